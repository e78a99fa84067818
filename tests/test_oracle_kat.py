"""The oracle's BVH builder against the reference's published known answers.

The reference publishes the uniform-SAH topology SHA-256 of its GI_TEST scene for leaf
sizes 1..64 (benchmarks/results/main-bvh-study/leaf-size-time.csv:2-8, hash domain of
gfxlab/benchmark/MethodCatalog.java:164-172), with node counts and depths.  Reproducing
them pins the C++ restatement of gfxlab/gpu/GpuScene.java's builder.
"""
import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode

GI_TEST_KAT = {
    1: ("466f59208c8732bd7b843b432e761ca2f75fac07083010682677d9cc4c5415ca", 7, 2),
    2: ("b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5", 3, 1),
    4: ("b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5", 3, 1),
    8: ("b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5", 3, 1),
    16: ("b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5", 3, 1),
    32: ("b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5", 3, 1),
    64: ("b824170b0cb427cbeb5f3d6c7502429645b650163fbd12bdba9b150d402e8ea5", 3, 1),
}


@pytest.mark.parametrize("leaf", sorted(GI_TEST_KAT))
def test_gi_test_topology_hash(leaf):
    sha, nodes, depth = GI_TEST_KAT[leaf]
    b = oracle.build_bvh(synth.gi_test_spheres(), BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, leaf))
    assert b.node_count == nodes
    assert b.max_depth == depth
    assert b.topology_sha256() == sha


def test_node_count_identity_and_leaf_rule():
    s = synth.hetero_scene(3000, 7, synth.WORKLOAD_IDS["test"], 0)
    b = oracle.build_bvh(s)
    assert b.node_count == 2 * b.leaf_count - b.root_count
    assert b.ref_count == s.bounded_primitive_count()
    assert sorted(b.refs.tolist()) == sorted(b.refs.tolist())
    nd = b.node_data.reshape(-1, 4)
    leaves = nd[nd[:, 0] < 0]
    assert leaves[:, 3].sum() == b.ref_count
    assert leaves[:, 3].max() <= 4  # leaf size 4 and no coincident centroids


def test_per_type_forest_roots():
    s = synth.hetero_scene(800, 3, synth.WORKLOAD_IDS["test"], 1)
    b = oracle.build_bvh(s, BvhBuildConfig.weighted(leaf_size=4, mode=BvhBuildMode.PER_TYPE_WEIGHTED_SAH))
    assert b.root_count == 4
    assert b.roots[0] == 0
    nd = b.node_data.reshape(-1, 4)
    kinds = set(nd[nd[:, 0] < 0, 0].tolist())
    assert -1 not in kinds  # per-type trees have homogeneous leaves only
