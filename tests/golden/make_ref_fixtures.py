"""Generates tests/golden/ref_trace_*.npz: closest-hit outputs of the reference's own CUDA
kernel (traceReplayKernel from gfxlab/gpu/GpuKernelSources.java, built for sm_100a by
oracle/build_oracle.py into oracle/_ref/), for the GI_TEST ray grid and the plain and
heterogeneous scenes, in both builds (NVRTC-default contraction and -fmad=false).

Run on a machine with an sm_100 GPU and oracle/_ref built:
    python tests/golden/make_ref_fixtures.py
The CPU test-suite checks the FP32 oracle against these recorded outputs.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "master-rad_b200"))

from oracle import oracle  # noqa: E402
from rtb200 import synth  # noqa: E402


def cases():
    gi_cam = synth.GpuCamera((0.0, 0.0, -3.0), (0.0, 0.0, 1.0), (0.41421356, 0.0, 0.0),
                             (0.0, 0.41421356, 0.0))
    yield "gi_test", synth.gi_test_scene(), synth.primary_grid(gi_cam, 32, 18)
    yield "plain", synth.plain_workload().scene, np.concatenate(
        [synth.primary_grid(synth.camera_looking_z((0.0, 0.0, -2.9)), 32, 18), synth.random_rays(2000, 5)])
    yield "hetero", synth.hetero_scene(2000, 11, synth.WORKLOAD_IDS["test"], 3), np.concatenate(
        [synth.primary_grid(synth.camera_looking_z((0.0, 0.0, -2.9)), 32, 18), synth.random_rays(3000, 6)])


def main(out_dir):
    for name, scene, rays in cases():
        bvh = oracle.build_bvh(scene)
        data = {"rays": rays}
        for variant in ("nofmad", "fmad"):
            r = oracle.ref_trace(scene, rays, bvh, variant=variant)
            for k in ("hit", "t", "order", "material", "normal"):
                data["%s_%s" % (variant, k)] = r[k]
        np.savez_compressed(os.path.join(out_dir, "ref_trace_%s.npz" % name), **data)
        print(name, len(rays), "rays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
