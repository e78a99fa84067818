"""The oracle's restatement of the reference's SBVH builder (SpatialBuildState,
gfxlab/gpu/GpuScene.java:1084-1412).

No SBVH tree of a reproducible scene is published by the reference (its SBVH rows are the
Hero scenes, built through a closed rotation library), so the restatement is pinned through
the parts it shares with the pinned object-SAH restatement: with the reference budget at
N (maxReferenceMultiplier 1) no spatial split is ever attempted, and on scenes whose
centroids are distinct per axis the SBVH recursion is the object-SAH recursion, so the GI_TEST
SBVH trees reproduce the published GI_TEST topology hashes and a 3,000-primitive scene
reproduces the full-sweep tree.  With the default budget the trees are checked for the
invariants of the format: every primitive referenced, leaf ranges tiling the references,
node count 2L - 1, and spatial splits only where duplicates appear."""
import numpy as np

from oracle import oracle
from rtb200 import synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode, BvhBuildOptions

GI_TEST = {1: "466f59208c8732bd7b843b432e761ca2f75fac07083010682677d9cc4c5415ca",
           4: "b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5"}


def test_sbvh_without_budget_reproduces_the_gi_test_hashes():
    for leaf, sha in GI_TEST.items():
        b = oracle.build_bvh_sbvh(synth.gi_test_spheres(),
                                  BvhBuildConfig(BvhBuildMode.UNIFORM_SBVH, leaf),
                                  BvhBuildOptions(max_reference_multiplier=1.0))
        assert b.topology_sha256() == sha
        assert b.spatial_splits == 0


def test_sbvh_without_budget_is_the_object_sah_tree():
    s = synth.hetero_scene(3000, 17, synth.WORKLOAD_IDS["test"], 60)
    for mode, sbvh in ((BvhBuildMode.UNIFORM_SAH, BvhBuildMode.UNIFORM_SBVH),
                       (BvhBuildMode.WEIGHTED_SAH, BvhBuildMode.WEIGHTED_SBVH)):
        cfg = BvhBuildConfig.weighted(leaf_size=4, mode=mode) if mode.uses_primitive_weights() \
            else BvhBuildConfig(mode, 4)
        scfg = BvhBuildConfig.weighted(leaf_size=4, mode=sbvh) if sbvh.uses_primitive_weights() \
            else BvhBuildConfig(sbvh, 4)
        want = oracle.build_bvh(s, cfg)
        got = oracle.build_bvh_sbvh(s, scfg, BvhBuildOptions(max_reference_multiplier=1.0))
        assert got.topology_sha256() == want.topology_sha256()
        assert (got.uniform_sah, got.weighted_sah, got.generalized_sah) == \
            (want.uniform_sah, want.weighted_sah, want.generalized_sah)


def test_sbvh_tree_invariants():
    s = synth.hetero_scene(2000, 19, synth.WORKLOAD_IDS["test"], 61)
    b = oracle.build_bvh_sbvh(s, BvhBuildConfig.weighted(leaf_size=4, mode=BvhBuildMode.WEIGHTED_SBVH))
    n = s.bounded_primitive_count()
    assert b.node_count == 2 * b.leaf_count - 1
    assert n <= b.ref_count <= 2 * n
    assert b.spatial_splits > 0 and b.ref_count > n  # the mix overlaps: some splits happen
    nd = b.node_data.reshape(-1, 4)
    leaves = nd[nd[:, 0] < 0]
    assert leaves[:, 3].sum() == b.ref_count
    order = np.argsort(leaves[:, 2])
    starts, counts = leaves[order, 2], leaves[order, 3]
    assert starts[0] == 0 and np.all(starts[1:] == starts[:-1] + counts[:-1])
    # every primitive appears; a part is split again only below depth maxSplitsPerPrimitive (8)
    idx = b.refs & 0x3FFFFFFF
    typ = (b.refs.astype(np.int64) >> 30) & 3
    keys = typ * (1 << 30) + idx
    uniq, mult = np.unique(keys, return_counts=True)
    assert len(uniq) == n
    assert mult.max() <= 2 ** 8
