"""The binned object-SAH device builder (rtb_scene_build_binned) against the oracle's CPU
restatement of the same binned rule, node for node, through the C ABI; plus the closest
hits over binned trees against linear traversal, and the SAH cost against the full sweep.

The binned mode has no reference counterpart (the reference builder is the full sweep of
gfxlab/gpu/GpuScene.java:1453-1488); its trees are compared with the oracle's binned
restatement, never with the Java tree."""
import numpy as np
import pytest

from oracle import oracle
from rtb200 import native, synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode, GpuScene, MaterialData
from rtb200.tracer import Context, ResidentScene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _check_binned(ctx, scene, cfg, bins):
    want = oracle.build_bvh(scene, cfg, bins=bins)
    rs = ResidentScene.build(ctx, scene, cfg, bins=bins)
    nb, nd, refs, roots = rs.download_bvh()
    st = rs.stats
    rs.close()
    np.testing.assert_array_equal(nb.view(np.int32), want.node_bounds.view(np.int32))
    np.testing.assert_array_equal(nd, want.node_data)
    np.testing.assert_array_equal(refs, want.refs)
    np.testing.assert_array_equal(roots, want.roots)
    assert (st.node_count, st.root_count, st.leaf_count, st.max_depth, st.primitive_ref_count) == \
        (want.node_count, want.root_count, want.leaf_count, want.max_depth, want.ref_count)
    assert (st.min_leaf_occupancy, st.max_leaf_occupancy) == (want.min_leaf, want.max_leaf)
    assert st.weighted_sah_cost == want.weighted_sah
    assert st.generalized_sah_cost == want.generalized_sah
    return st


def _cfg(mode, leaf):
    return BvhBuildConfig.weighted(leaf_size=leaf, mode=mode) if mode.uses_primitive_weights() \
        else BvhBuildConfig(mode, leaf)


@pytest.mark.parametrize("mode", [BvhBuildMode.UNIFORM_SAH, BvhBuildMode.WEIGHTED_SAH,
                                  BvhBuildMode.PER_TYPE_SAH, BvhBuildMode.PER_TYPE_WEIGHTED_SAH])
@pytest.mark.parametrize("bins", [2, 16, 32])
@pytest.mark.parametrize("n", [7, 129, 3000])
def test_binned_identical_to_oracle(ctx, mode, bins, n):
    scene = synth.hetero_scene(n, 500 + n, synth.WORKLOAD_IDS["test"], 3)
    _check_binned(ctx, scene, _cfg(mode, 4), bins)


@pytest.mark.parametrize("leaf", [1, 2, 8])
def test_binned_leaf_sizes(ctx, leaf):
    scene = synth.hetero_scene(2000, 41, synth.WORKLOAD_IDS["test"], 4)
    _check_binned(ctx, scene, _cfg(BvhBuildMode.WEIGHTED_SAH, leaf), 32)


def test_binned_bench_workloads(ctx):
    _check_binned(ctx, synth.plain_workload().scene, synth.plain_workload().scene.config, 16)
    h = synth.hetero_workload().scene
    st = _check_binned(ctx, h, h.config, 32)
    full = oracle.build_bvh(h)
    # binned splits see only bin boundaries: a little above the full sweep's cost
    assert full.generalized_sah <= st.generalized_sah_cost <= 1.05 * full.generalized_sah


def test_binned_degenerate_inputs(ctx):
    m = MaterialData.matte((0.5, 0.5, 0.5))
    # coincident centroids in a node above the one-warp size: median splits in input order
    s = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 2))
    for _ in range(300):
        s.add_sphere((0.25, -0.5, 1.0), 0.3, m)
    for k in range(20):
        s.add_box((k, 0, 0), (k + 0.5, 0.5, 0.5), m)
    st = _check_binned(ctx, s, s.config, 32)
    assert st.max_leaf_occupancy <= 2
    # coincident centroids within the leaf size: one leaf
    s0 = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 8))
    for _ in range(5):
        s0.add_sphere((0.0, 0.0, 0.0), 0.5, m)
    st = _check_binned(ctx, s0, s0.config, 8)
    assert st.node_count == 1
    # single primitive, and centroids spread along one axis only
    s1 = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 4))
    s1.add_box((0, 0, 0), (1, 1, 1), m)
    _check_binned(ctx, s1, s1.config, 4)
    s2 = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 1))
    for k in range(400):
        s2.add_sphere((0.0, 0.05 * k, 0.0), 0.01 + 0.001 * (k % 3), m)
    _check_binned(ctx, s2, s2.config, 32)


def _trace(ctx, rs, rays, use_bvh):
    import ctypes as C  # noqa: F401
    n = len(rays)
    out = dict(hit=np.zeros(n, np.int32), t=np.zeros(n, np.float32), order=np.zeros(n, np.int32),
               material=np.zeros(n, np.int32), normal=np.zeros(3 * n, np.float32))
    r = native.f32(rays).reshape(-1)
    ctx.check(ctx.lib.rtb_trace_replay(ctx.handle, rs.handle, native.fptr(r), n, 1 if use_bvh else 0,
                                       0, native.iptr(out["hit"]), native.fptr(out["t"]),
                                       native.iptr(out["order"]), native.iptr(out["material"]),
                                       native.fptr(out["normal"])))
    return out


def test_binned_hits_equal_linear_and_oracle(ctx):
    w = synth.hetero_workload()
    rays = np.concatenate([synth.primary_grid(w.camera, 48, 48), synth.random_rays(4000, 11)])
    rs = ResidentScene.build(ctx, w.scene, bins=32)
    bvh = _trace(ctx, rs, rays, True)
    lin = _trace(ctx, rs, rays, False)
    rs.close()
    ref = oracle.trace(w.scene, rays, oracle.build_bvh(w.scene, bins=32), use_bvh=True)
    for k in ("hit", "order", "material"):
        np.testing.assert_array_equal(bvh[k], lin[k])
    np.testing.assert_array_equal(bvh["t"].view(np.int32), lin["t"].view(np.int32))
    np.testing.assert_array_equal(bvh["normal"].view(np.int32), lin["normal"].view(np.int32))
    np.testing.assert_array_equal(bvh["order"], ref["order"])
    np.testing.assert_array_equal(bvh["t"].view(np.int32), np.asarray(ref["t"], np.float32).view(np.int32))


def test_binned_rejects_bad_bin_counts(ctx):
    scene = synth.hetero_scene(50, 1, synth.WORKLOAD_IDS["test"], 2)
    for bins in (1, 33, -4):
        with pytest.raises(ValueError, match="2..32 bins"):
            ResidentScene.build(ctx, scene, bins=bins)


@pytest.mark.slow
def test_binned_one_million_identical(ctx):
    w = synth.scale_workload()
    st = _check_binned(ctx, w.scene, w.scene.config, 32)
    assert st.primitive_ref_count == 1_000_001
