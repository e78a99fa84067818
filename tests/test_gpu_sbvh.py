"""The library's SBVH builder (rtb_scene_build with modes UNIFORM_SBVH / WEIGHTED_SBVH,
through the C ABI) against the oracle's restatement of the reference's SpatialBuildState
(gfxlab/gpu/GpuScene.java:1084-1412), node for node: the flattened arrays (float bounds bit
for bit, node data, references with their duplicates, roots), BvhStats counts, the three SAH
costs, the spatial split count and the duplicate count.  A scene resident with an SBVH tree
traces exactly as with no tree at all (duplicated references and clipped node bounds never
change a closest hit)."""
import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode, BvhBuildOptions
from rtb200.tracer import Context, ResidentScene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _cfg(mode, leaf):
    return BvhBuildConfig.weighted(leaf_size=leaf, mode=mode) if mode.uses_primitive_weights() \
        else BvhBuildConfig(mode, leaf)


def _identical(ctx, scene, cfg, options):
    scene.options = options
    want = oracle.build_bvh_sbvh(scene, cfg, options)
    rs = ResidentScene.build(ctx, scene, cfg)
    nb, nd, refs, roots = rs.download_bvh()
    st = rs.stats
    rs.close()
    np.testing.assert_array_equal(nb.view(np.int32), want.node_bounds.view(np.int32))
    np.testing.assert_array_equal(nd, want.node_data)
    np.testing.assert_array_equal(refs, want.refs)
    np.testing.assert_array_equal(roots, want.roots)
    assert (st.node_count, st.leaf_count, st.max_depth, st.primitive_ref_count) == \
        (want.node_count, want.leaf_count, want.max_depth, want.ref_count)
    assert (st.min_leaf_occupancy, st.max_leaf_occupancy) == (want.min_leaf, want.max_leaf)
    assert (st.uniform_sah_cost, st.weighted_sah_cost, st.generalized_sah_cost) == \
        (want.uniform_sah, want.weighted_sah, want.generalized_sah)
    assert st.spatial_split_count == want.spatial_splits
    assert st.duplicate_reference_count == want.ref_count - scene.bounded_primitive_count()
    return st


@pytest.mark.parametrize("mode", [BvhBuildMode.UNIFORM_SBVH, BvhBuildMode.WEIGHTED_SBVH])
@pytest.mark.parametrize("leaf", [1, 4])
@pytest.mark.parametrize("n", [40, 1500, 6000])
def test_sbvh_identical_to_restatement(ctx, mode, leaf, n):
    scene = synth.hetero_scene(n, 900 + n, synth.WORKLOAD_IDS["test"], 70 + leaf)
    st = _identical(ctx, scene, _cfg(mode, leaf), BvhBuildOptions())
    if n >= 1500:
        assert st.spatial_split_count > 0


@pytest.mark.parametrize("opts", [BvhBuildOptions(spatial_bins=8, max_reference_multiplier=1.2),
                                  BvhBuildOptions(max_splits_per_primitive=1, min_spatial_references=4),
                                  BvhBuildOptions(spatial_overlap_threshold=0.0, spatial_bins=33)],
                         ids=["8-bins-budget-1.2", "one-split-per-primitive", "no-overlap-threshold"])
def test_sbvh_options(ctx, opts):
    scene = synth.hetero_scene(2500, 77, synth.WORKLOAD_IDS["test"], 80)
    _identical(ctx, scene, _cfg(BvhBuildMode.WEIGHTED_SBVH, 4), opts)


def test_sbvh_benchmark_scene(ctx):
    """The heterogeneous 10k benchmark scene, weighted SBVH with the default options."""
    w = synth.hetero_workload()
    st = _identical(ctx, w.scene, _cfg(BvhBuildMode.WEIGHTED_SBVH, 4), BvhBuildOptions())
    print("\nSBVH 10k: %d nodes, %d references (%d duplicates), %d spatial splits, %.1f ms"
          % (st.node_count, st.primitive_ref_count, st.duplicate_reference_count,
             st.spatial_split_count, st.build_ms))


def test_sbvh_tree_traces_like_linear(ctx):
    import ctypes as C
    from rtb200 import native as N
    scene = synth.hetero_scene(3000, 55, synth.WORKLOAD_IDS["test"], 81)
    scene.options = BvhBuildOptions()
    rs = ResidentScene.build(ctx, scene, _cfg(BvhBuildMode.WEIGHTED_SBVH, 4))
    cam = synth.camera_looking_z((0.0, 0.0, -2.9))
    rays = np.concatenate([synth.primary_grid(cam, 64, 48), synth.random_rays(4000, 56)])
    n = len(rays)
    outs = []
    for use_bvh in (1, 0):
        o = [np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros(n, np.int32),
             np.zeros(n, np.int32), np.zeros(3 * n, np.float32)]
        r = N.f32(rays).reshape(-1)
        ctx.check(ctx.lib.rtb_trace_replay(ctx.handle, rs.handle, N.fptr(r), n, use_bvh, 0,
                                           N.iptr(o[0]), N.fptr(o[1]), N.iptr(o[2]),
                                           N.iptr(o[3]), N.fptr(o[4])))
        outs.append(o)
    rs.close()
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))
    assert outs[0][0].sum() > 0
