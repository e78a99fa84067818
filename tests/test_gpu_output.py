"""Grid-material planes on the device against the reference kernel and the oracle (closest
hits, materials and normals bit for bit; a rendered frame bit for bit), and the headless
renderer's multi-frame accumulation, tonemap and PNG output over the device renderer."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle
from rtb200 import image as I
from rtb200 import synth
from rtb200.tracer import GpuRayTracer

from test_image_output import grid_rays, grid_scene

pytestmark = pytest.mark.gpu


def _same(a, b):
    np.testing.assert_array_equal(np.asarray(a["hit"]), np.asarray(b["hit"]))
    np.testing.assert_array_equal(np.asarray(a["order"]), np.asarray(b["order"]))
    np.testing.assert_array_equal(np.asarray(a["material"]), np.asarray(b["material"]))
    np.testing.assert_array_equal(np.asarray(a["t"], np.float32).view(np.int32),
                                  np.asarray(b["t"], np.float32).view(np.int32))
    np.testing.assert_array_equal(np.asarray(a["normal"], np.float32).reshape(-1, 3).view(np.int32),
                                  np.asarray(b["normal"], np.float32).reshape(-1, 3).view(np.int32))


def test_grid_plane_hits_match_reference_kernel():
    s = grid_scene()
    rays = grid_rays()
    bvh = oracle.build_bvh(s)
    with GpuRayTracer(8, 8, 1) as tr:
        r = tr.trace_replay(s, rays)
    ours = {"hit": r.hit_flags, "t": r.hit_distances, "order": r.hit_primitive_orders,
            "material": r.hit_material_indices, "normal": r.hit_normals}
    ref = oracle.ref_trace(s, rays, bvh, variant="nofmad")
    _same(ours, ref)
    _same(ours, oracle.trace(s, rays, bvh))
    assert len(set(np.asarray(r.hit_material_indices).tolist())) >= 3


def test_grid_plane_render_matches_reference_kernel():
    s = grid_scene()
    cam = synth.camera_looking_z((0.0, 0.9, -2.5))
    w = synth.Workload("grid", s, cam, 96, 96, 4, 5, frame_seed=7, frame_index=2)
    with GpuRayTracer(w.width, w.height, w.spp) as tr:
        img = tr.render_sample(None, s, cam, w.max_depth, w.frame_index, w.frame_seed).reshape(-1, 3)
    ref, _ = oracle.ref_render(w, oracle.build_bvh(s), variant="nofmad")
    np.testing.assert_array_equal(img.view(np.int32), ref.view(np.int32))


def test_accumulated_frames_tonemap_and_png(tmp_path):
    w = dataclasses.replace(synth.plain_workload(), width=64, height=48, spp=2)
    with GpuRayTracer(w.width, w.height, w.spp) as tr:
        img = I.render_frames(tr, w.scene, w.camera, w.max_depth, frames=3, warmup_frames=1, seed=5)
        # the accumulated sums are the three measured frames times the samples per frame
        frames = [tr.render_sample(None, w.scene, w.camera, w.max_depth, i, I.frame_seed(5, i))
                  for i in (1, 2, 3)]
    want = sum(f.astype(np.float64) * w.spp for f in frames)
    np.testing.assert_array_equal(img.sums, want)
    assert img.samples == 6
    p = img.write_png(tmp_path / "plain.png")
    px = I.decode_png(p.read_bytes())
    assert px.shape == (48, 64, 4) and px[..., :3].max() > 0
