"""Tree identity of the device BVH builder against the oracle's restatement of the Java
builder (gfxlab/gpu/GpuScene.java:614-838, 1414-1499), through the C ABI.

"Identical" means the flattened arrays a Java caller would get from GpuScene --
bvhNodeBoundsData (bit for bit), bvhNodeData, bvhPrimitiveRefs, bvhRootIndices -- and so the
same MethodCatalog.topologySha256; BvhStats node/leaf/depth/occupancy counts and the three
SAH costs must be equal too.
"""
import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode, GpuScene, MaterialData
from rtb200.tracer import Context, ResidentScene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _check_identical(ctx, scene, cfg):
    want = oracle.build_bvh(scene, cfg)
    rs = ResidentScene.build(ctx, scene, cfg)
    nb, nd, refs, roots = rs.download_bvh()
    st = rs.stats
    rs.close()
    np.testing.assert_array_equal(nb.view(np.int32), want.node_bounds.view(np.int32))
    np.testing.assert_array_equal(nd, want.node_data)
    np.testing.assert_array_equal(refs, want.refs)
    np.testing.assert_array_equal(roots, want.roots)
    assert oracle.topology_sha256(nb, nd, refs, roots) == want.topology_sha256()
    assert (st.node_count, st.root_count, st.leaf_count, st.max_depth, st.primitive_ref_count) == \
        (want.node_count, want.root_count, want.leaf_count, want.max_depth, want.ref_count)
    assert (st.min_leaf_occupancy, st.max_leaf_occupancy) == (want.min_leaf, want.max_leaf)
    assert st.uniform_sah_cost == want.uniform_sah
    assert st.weighted_sah_cost == want.weighted_sah
    assert st.generalized_sah_cost == want.generalized_sah
    return st


GI_TEST_KAT = {1: "466f59208c8732bd7b843b432e761ca2f75fac07083010682677d9cc4c5415ca",
               2: "b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5",
               8: "b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5",
               64: "b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5"}


@pytest.mark.parametrize("leaf", sorted(GI_TEST_KAT))
def test_device_build_reproduces_gi_test_hashes(ctx, leaf):
    rs = ResidentScene.build(ctx, synth.gi_test_scene(), BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, leaf))
    assert oracle.topology_sha256(*rs.download_bvh()) == GI_TEST_KAT[leaf]
    rs.close()


@pytest.mark.parametrize("mode", [BvhBuildMode.UNIFORM_SAH, BvhBuildMode.WEIGHTED_SAH,
                                  BvhBuildMode.PER_TYPE_SAH, BvhBuildMode.PER_TYPE_WEIGHTED_SAH])
@pytest.mark.parametrize("leaf", [1, 2, 4, 8])
@pytest.mark.parametrize("n", [7, 300, 5000])
def test_device_build_identical(ctx, mode, leaf, n):
    scene = synth.hetero_scene(n, 100 + n, synth.WORKLOAD_IDS["test"], leaf)
    cfg = BvhBuildConfig.weighted(leaf_size=leaf, mode=mode) if mode.uses_primitive_weights() \
        else BvhBuildConfig(mode, leaf)
    _check_identical(ctx, scene, cfg)


def test_device_build_plain_and_hetero_workloads(ctx):
    for w in (synth.plain_workload(), synth.hetero_workload()):
        st = _check_identical(ctx, w.scene, w.scene.config)
        # weighted nodes above the sequential size take certified count-based weights; only
        # a few need the sequential order
        print("\n%s: %d nodes, %d summed sequentially after certification failed"
              % (w.name, st.node_count, st.sequential_nodes))
        assert st.sequential_nodes <= max(2, st.node_count // 100)


def test_certified_weights_fall_back_on_exact_ties(ctx):
    """A mirror-symmetric row of 1,201 spheres and boxes (dyadic positions centred on 0, a
    palindromic type pattern): the two middle splits cost the same in exact arithmetic, so
    the count-based weights cannot tell which one the reference's sequential rounding
    prefers.  Those nodes fail certification and take the sequential weights; the tree is
    still the reference's."""
    n = 1201
    i = np.arange(n)
    x = (i - (n - 1) / 2) / 8.0
    kind = np.minimum(i, n - 1 - i) % 3
    s = GpuScene(BvhBuildConfig.weighted(leaf_size=4))
    mid = s.register_material(MaterialData.matte((0.5, 0.5, 0.5)))
    c = np.stack([x, np.zeros(n), np.zeros(n)], axis=1)
    sp = kind == 0
    s.add_spheres(c[sp], np.full(sp.sum(), 0.05), np.full(sp.sum(), mid))
    s.add_boxes(c[~sp] - 0.05, c[~sp] + 0.05, np.full((~sp).sum(), mid))
    st = _check_identical(ctx, s, s.config)
    print("\nsymmetric row: %d nodes, %d sequential" % (st.node_count, st.sequential_nodes))
    assert st.sequential_nodes >= 1


def test_device_build_calibrated_weights(ctx):
    """The reference's calibrated RTX 3080 weights (PrimitiveCostModel.java:11-19), lambda 0.5."""
    scene = synth.hetero_scene(4000, 77, synth.WORKLOAD_IDS["test"], 9)
    cfg = BvhBuildConfig(BvhBuildMode.WEIGHTED_SAH, 4, lam=0.5)
    _check_identical(ctx, scene, cfg)


def test_device_build_degenerate_inputs(ctx):
    m = MaterialData.matte((0.5, 0.5, 0.5))
    # coincident centroids: no split axis exists, one oversized leaf (GpuScene.java:1435-1436)
    s = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 2))
    for _ in range(5):
        s.add_sphere((0.25, -0.5, 1.0), 0.3, m)
    st = _check_identical(ctx, s, s.config)
    assert st.max_leaf_occupancy == 5
    # single primitive
    s1 = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 4))
    s1.add_box((0, 0, 0), (1, 1, 1), m)
    _check_identical(ctx, s1, s1.config)
    # equal centroids on one axis only
    s2 = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 1))
    for k in range(40):
        s2.add_sphere((0.0, 0.05 * k, 0.0), 0.01 + 0.001 * (k % 3), m)
    _check_identical(ctx, s2, s2.config)


def test_binned_build_rejects_the_sbvh_modes(ctx):
    """The SBVH modes have their own builder (tests/test_gpu_sbvh.py); the binned object-SAH
    builder refuses them."""
    scene = synth.hetero_scene(50, 1, synth.WORKLOAD_IDS["test"], 2)
    from rtb200 import native
    with pytest.raises(native.RtbError) as e:
        ResidentScene.build(ctx, scene, BvhBuildConfig(BvhBuildMode.UNIFORM_SBVH, 4), bins=16)
    assert e.value.status == 5


@pytest.mark.slow
def test_device_build_one_million_identical(ctx):
    w = synth.scale_workload()
    st = _check_identical(ctx, w.scene, w.scene.config)
    assert st.primitive_ref_count == 1_000_001
    print("\n1M: %d nodes, %d summed sequentially after certification failed, build %.1f ms"
          % (st.node_count, st.sequential_nodes, st.build_ms))
    assert st.sequential_nodes <= st.node_count // 100


@pytest.mark.slow
def test_device_build_identical_beyond_one_tile_of_chunks(ctx):
    """1.2M primitives: more than 1,024 scan chunks of 1,024 positions, so the segmented
    scans carry their chunk aggregates across two tiles of the carry kernel (the root node
    of the first level spans every chunk of both tiles)."""
    w = synth.scale_workload(n=1_200_000)
    st = _check_identical(ctx, w.scene, w.scene.config)
    assert st.primitive_ref_count == 1_200_001
    assert (st.primitive_ref_count + 1023) // 1024 > 1024


@pytest.mark.parametrize("mode", [BvhBuildMode.SAH_ROTATIONS, BvhBuildMode.WEIGHTED_SAH_ROTATIONS])
@pytest.mark.parametrize("n", [7, 300, 5000])
def test_device_rotation_modes_identical(ctx, mode, n):
    """BvhRotator (GpuScene.java:968-1057) after the device SAH build: the same rotated tree
    as the oracle's restatement, node for node, and the same rotation count."""
    scene = synth.hetero_scene(n, 300 + n, synth.WORKLOAD_IDS["test"], 5)
    cfg = BvhBuildConfig.weighted(leaf_size=4, mode=mode) if mode.uses_primitive_weights() \
        else BvhBuildConfig(mode, 4)
    st = _check_identical(ctx, scene, cfg)
    assert st.rotation_count == oracle.build_bvh(scene, cfg).rotations


def test_device_rotation_passes_option(ctx):
    from rtb200.scene import BvhBuildOptions
    w = synth.hetero_workload()
    cfg = BvhBuildConfig.weighted(leaf_size=4, mode=BvhBuildMode.WEIGHTED_SAH_ROTATIONS)
    for passes in (1, 2):
        want = oracle.build_bvh(w.scene, cfg, rotation_passes=passes)
        w.scene.options = BvhBuildOptions(rotation_passes=passes)
        rs = ResidentScene.build(ctx, w.scene, cfg)
        assert oracle.topology_sha256(*rs.download_bvh()) == want.topology_sha256()
        assert rs.stats.rotation_count == want.rotations
        rs.close()
    w.scene.options = BvhBuildOptions()
