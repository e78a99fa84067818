"""CPU checks of the oracle's BvhRotator restatement (gfxlab/gpu/GpuScene.java:968-1057): the
rotation modes keep the SAH tree's leaves and lower its area cost, pass by pass."""
import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode


def _cfg(mode, leaf=4):
    return BvhBuildConfig.weighted(leaf_size=leaf, mode=mode) if mode.uses_primitive_weights() \
        else BvhBuildConfig(mode, leaf)


@pytest.mark.parametrize("mode,base", [(BvhBuildMode.SAH_ROTATIONS, BvhBuildMode.UNIFORM_SAH),
                                       (BvhBuildMode.WEIGHTED_SAH_ROTATIONS, BvhBuildMode.WEIGHTED_SAH)])
def test_rotations_lower_the_cost_and_keep_the_leaves(mode, base):
    scene = synth.hetero_scene(3000, 21, synth.WORKLOAD_IDS["test"], 7)
    b0 = oracle.build_bvh(scene, _cfg(base))
    b1 = oracle.build_bvh(scene, _cfg(mode))
    assert b1.rotations > 0
    assert b1.generalized_sah <= b0.generalized_sah * (1 + 1e-12)
    assert (b1.node_count, b1.leaf_count, b1.ref_count) == (b0.node_count, b0.leaf_count, b0.ref_count)
    assert sorted(b1.refs.tolist()) == sorted(b0.refs.tolist())
    # leaf sizes are a multiset property of the unchanged leaves
    def leaf_sizes(b):
        nd = b.node_data.reshape(-1, 4)
        return sorted(nd[nd[:, 1] < 0, 3].tolist())
    assert leaf_sizes(b1) == leaf_sizes(b0)
    # more passes never raise the cost; one pass makes fewer or equal rotations
    b_one = oracle.build_bvh(scene, _cfg(mode), rotation_passes=1)
    assert b_one.rotations <= b1.rotations
    assert b1.generalized_sah <= b_one.generalized_sah * (1 + 1e-12)
    assert oracle.build_bvh(scene, _cfg(mode)).topology_sha256() == b1.topology_sha256()


def test_rotation_passes_must_be_positive():
    scene = synth.hetero_scene(50, 2, synth.WORKLOAD_IDS["test"], 1)
    with pytest.raises(RuntimeError):
        oracle.build_bvh(scene, _cfg(BvhBuildMode.SAH_ROTATIONS), rotation_passes=0)
