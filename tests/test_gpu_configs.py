"""Parity at the benchmark configurations themselves, whole frames at full size.

* C1 plain: 64 spheres and an emitter in a closed room, 256x256, 16 spp, depth 4, uniform
  SAH with leaves of at most 4.
* C2 heterogeneous: 10,000 mixed primitives (spheres, boxes, affine spheres, affine boxes),
  1024x1024, 64 spp, depth 8, weighted SAH (sphere 1.0, box 1.3, affine 2.1).
* C3 scale: 1,000,000 primitives of the same mix in 64 Gaussian clusters, 1920x1080,
  256 spp, depth 8.

Each frame is rendered through the C ABI from the tree the device builder made and
compared with the reference's own renderKernel (gfxlab/gpu/GpuKernelSources.java:1167-1315)
launched with renderSample's tile plan (gfxlab/gpu/GpuRayTracer.java:317-432) on the same
tree, seeds and camera:

* built without contraction, the reference image is equal bit for bit;
* built as NVRTC builds it (contraction on, the reference's default), the per-pixel relative
  error is within 1e-4 except at pixels where a path flips at a contraction-sensitive near
  tie; the share of such pixels is bounded at 0.1 % (the C2 bench frame measures about
  0.04 %).

Closest hits on the C2 scene itself (primary grid of the bench camera at full resolution
plus random rays) are bit-identical to traceReplayKernel built without contraction; against
the contracting build a differing primitive is accepted only when, in one arithmetic (the
oracle's uncontracted FP32), its distance is within 1e-6 relative of this library's hit.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from rtb200 import native as N
from rtb200 import synth
from rtb200.tracer import Context, ResidentScene, camera_struct

pytestmark = pytest.mark.gpu

NEAR_TIE_REL = 1e-6
PIXEL_REL = 1e-4
OUTLIER_SHARE = 1e-3


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _workload(name):
    if name == "C1":
        return synth.plain_workload()
    if name == "C2":
        return synth.hetero_workload()
    return synth.scale_workload()


class _Tree:
    def __init__(self, arrays):
        self.node_bounds, self.node_data, self.refs, self.roots = arrays
        self.node_count = len(self.node_data) // 4
        self.ref_count = len(self.refs)
        self.root_count = len(self.roots)


def _render_device(ctx, w):
    """Device build + one frame through rtb_render_sample into a host buffer; returns the
    image and the device tree in the reference's flattened layout."""
    res = ResidentScene.build(ctx, w.scene)
    try:
        img = np.zeros(w.width * w.height * 3, np.float32)
        p = N.RenderParams(w.width, w.height, w.spp, w.max_depth, w.frame_index,
                           w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
        cam = camera_struct(w.camera)
        ctx.check(ctx.lib.rtb_render_sample(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                            N.fptr(img)))
        tree = _Tree(res.download_bvh())
    finally:
        res.close()
    return img.reshape(-1, 3), tree


_frames = {}


def _frame(ctx, name):
    if name not in _frames:
        w = _workload(name)
        img, tree = _render_device(ctx, w)
        _frames[name] = (w, img, tree)
    return _frames[name]


@pytest.mark.skipif(not oracle.ref_available("nofmad"), reason="reference kernel not built")
@pytest.mark.parametrize("name", ["C1", "C2", "C3"])
def test_config_frame_bit_identical_to_reference_kernel(ctx, name):
    w, dev, tree = _frame(ctx, name)
    if name != "C3":
        # the device tree is the reference builder's (the 1M tree is compared in
        # test_gpu_build.py); here the hash of the whole flattened tree
        want = oracle.build_bvh(w.scene)
        assert oracle.topology_sha256(tree.node_bounds, tree.node_data, tree.refs, tree.roots) \
            == want.topology_sha256()
    ref, ms = oracle.ref_render(w, tree, variant="nofmad")
    same = np.all(dev.view(np.int32) == ref.view(np.int32), axis=1)
    print("\n%s %dx%d %d spp depth %d: %d of %d pixels bit-identical; reference kernel %.0f ms"
          % (name, w.width, w.height, w.spp, w.max_depth, int(same.sum()), len(same), ms))
    np.testing.assert_array_equal(dev.view(np.int32), ref.view(np.int32))


@pytest.mark.skipif(not oracle.ref_available("fmad"), reason="reference kernel not built")
@pytest.mark.parametrize("name", ["C1", "C2"])
def test_config_frame_vs_reference_kernel_as_shipped(ctx, name):
    w, dev, tree = _frame(ctx, name)
    ref, _ = oracle.ref_render(w, tree, variant="fmad")
    rel = np.abs(dev.astype(np.float64) - ref) / np.maximum(np.abs(ref.astype(np.float64)), 1e-3)
    per_pixel = rel.max(axis=1)
    share = float((per_pixel > PIXEL_REL).mean())
    print("\n%s vs contracting build: %.4f %% of pixels above %.0e relative, median %.2e, "
          "max %.3g" % (name, 100 * share, PIXEL_REL, float(np.median(per_pixel)),
                        float(per_pixel.max())))
    assert np.median(per_pixel) <= PIXEL_REL
    assert share <= OUTLIER_SHARE


def _trace(ctx, res, rays, use_bvh=True):
    n = len(rays)
    out = dict(hit=np.zeros(n, np.int32), t=np.zeros(n, np.float32), order=np.zeros(n, np.int32),
               material=np.zeros(n, np.int32), normal=np.zeros(3 * n, np.float32))
    r = N.f32(rays).reshape(-1)
    ctx.check(ctx.lib.rtb_trace_replay(ctx.handle, res.handle, N.fptr(r), n, 1 if use_bvh else 0,
                                       0, N.iptr(out["hit"]), N.fptr(out["t"]),
                                       N.iptr(out["order"]), N.iptr(out["material"]),
                                       N.fptr(out["normal"])))
    out["normal"] = out["normal"].reshape(-1, 3)
    return out


def _c2_rays():
    w = synth.hetero_workload()
    grid = synth.primary_grid(w.camera, w.width, w.height)
    rnd = synth.random_rays(200000, 9)
    return w, np.concatenate([grid, rnd])


def _assert_identical(a, b):
    np.testing.assert_array_equal(a["hit"], b["hit"])
    np.testing.assert_array_equal(a["order"], b["order"])
    np.testing.assert_array_equal(a["material"], b["material"])
    np.testing.assert_array_equal(a["t"].view(np.int32), b["t"].view(np.int32))
    np.testing.assert_array_equal(a["normal"].view(np.int32), b["normal"].view(np.int32))


@pytest.mark.skipif(not oracle.ref_available("nofmad"), reason="reference kernel not built")
def test_c2_trace_bit_identical_to_reference_kernel(ctx):
    w, rays = _c2_rays()
    res = ResidentScene.build(ctx, w.scene)
    try:
        tree = _Tree(res.download_bvh())
        dev = _trace(ctx, res, rays)
    finally:
        res.close()
    ref = oracle.ref_trace(w.scene, rays, tree, variant="nofmad")
    _assert_identical(dev, ref)
    # the FP32 restatement agrees on a slice (it runs on one host core)
    cpu = oracle.trace(w.scene, rays[::50], tree)
    _assert_identical({k: v[::50] for k, v in dev.items()}, cpu)


@pytest.mark.skipif(not oracle.ref_available("fmad"), reason="reference kernel not built")
def test_c2_trace_vs_reference_kernel_as_shipped_near_ties_only(ctx):
    w, rays = _c2_rays()
    res = ResidentScene.build(ctx, w.scene)
    try:
        tree = _Tree(res.download_bvh())
        dev = _trace(ctx, res, rays)
    finally:
        res.close()
    ref = oracle.ref_trace(w.scene, rays, tree, variant="fmad")
    np.testing.assert_array_equal(dev["hit"], ref["hit"])
    bad = np.nonzero(dev["order"] != ref["order"])[0]
    # the contracting build's winner, measured in the uncontracted arithmetic that picked
    # ours: a near tie of our hit, or the pick would be a real disagreement
    alt = oracle.primitive_distance(w.scene, rays[bad], ref["order"][bad])
    t_dev = dev["t"][bad].astype(np.float64)
    gap = np.abs(alt.astype(np.float64) - t_dev) / np.abs(t_dev)
    print("\nC2 trace vs contracting build: %d of %d primitive ids differ; largest gap %.3g"
          % (len(bad), len(rays), float(gap.max()) if len(bad) else 0.0))
    assert np.all(gap < NEAR_TIE_REL), gap.max()
    assert len(bad) <= max(1, len(rays) // 1000)
    hit = dev["hit"] == 1
    rel = np.abs(dev["t"][hit] - ref["t"][hit]) / np.maximum(1.0, np.abs(ref["t"][hit]))
    assert rel.max() < 1e-4  # the correctness gate's distance tolerance
