"""The FP32 oracle against the reference kernel's own recorded outputs (CPU only).

tests/golden/ref_trace_*.npz hold traceReplayKernel outputs of the reference's CUDA source
(gfxlab/gpu/GpuKernelSources.java, compiled for sm_100a by oracle/build_oracle.py) on the
GI_TEST primary grid and on the plain and heterogeneous scenes, generated by
tests/golden/make_ref_fixtures.py.  The oracle restates the kernel without contraction, so
against the -fmad=false build it must agree bit for bit; against the NVRTC-default build ids
may differ only at near ties.
"""
import os

import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _scene(name):
    if name == "gi_test":
        return synth.gi_test_scene()
    if name == "plain":
        return synth.plain_workload().scene
    return synth.hetero_scene(2000, 11, synth.WORKLOAD_IDS["test"], 3)


@pytest.mark.parametrize("name", ["gi_test", "plain", "hetero"])
def test_oracle_equals_reference_kernel_without_contraction(name):
    data = np.load(os.path.join(HERE, "ref_trace_%s.npz" % name))
    scene = _scene(name)
    rays = data["rays"]
    got = oracle.trace(scene, rays, oracle.build_bvh(scene))
    np.testing.assert_array_equal(got["hit"], data["nofmad_hit"])
    np.testing.assert_array_equal(got["order"], data["nofmad_order"])
    np.testing.assert_array_equal(got["material"], data["nofmad_material"])
    np.testing.assert_array_equal(got["t"].view(np.int32), data["nofmad_t"].view(np.int32))
    np.testing.assert_array_equal(got["normal"].view(np.int32), data["nofmad_normal"].view(np.int32))


@pytest.mark.parametrize("name", ["gi_test", "plain", "hetero"])
def test_oracle_vs_reference_kernel_as_shipped(name):
    data = np.load(os.path.join(HERE, "ref_trace_%s.npz" % name))
    scene = _scene(name)
    got = oracle.trace(scene, data["rays"], oracle.build_bvh(scene))
    np.testing.assert_array_equal(got["hit"], data["fmad_hit"])
    differ = got["order"] != data["fmad_order"]
    assert differ.sum() <= max(1, len(differ) // 1000)
    hit = got["hit"] == 1
    rel = np.abs(got["t"][hit] - data["fmad_t"][hit]) / np.maximum(1.0, np.abs(data["fmad_t"][hit]))
    assert rel.max() < 1e-4  # the reference correctness gate's distance tolerance


def test_linear_mode_equals_bvh_mode_on_fixture_rays():
    data = np.load(os.path.join(HERE, "ref_trace_hetero.npz"))
    scene = _scene("hetero")
    a = oracle.trace(scene, data["rays"], oracle.build_bvh(scene))
    b = oracle.trace(scene, data["rays"], None, use_bvh=False)
    np.testing.assert_array_equal(a["order"], b["order"])
    np.testing.assert_array_equal(a["t"].view(np.int32), b["t"].view(np.int32))
