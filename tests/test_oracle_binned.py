"""CPU checks of the oracle's binned object-SAH restatement (the rule the device's binned
builder follows): structural invariants, determinism, and its cost against the full sweep."""
import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode, GpuScene, MaterialData


def _leaf_sizes(b):
    nd = b.node_data.reshape(-1, 4)
    return nd[nd[:, 1] < 0, 3] if len(nd) else np.zeros(0, np.int32)


@pytest.mark.parametrize("bins", [2, 16, 32])
@pytest.mark.parametrize("mode", [BvhBuildMode.UNIFORM_SAH, BvhBuildMode.PER_TYPE_WEIGHTED_SAH])
def test_binned_structure(bins, mode):
    scene = synth.hetero_scene(1500, 3, synth.WORKLOAD_IDS["test"], 5)
    cfg = BvhBuildConfig.weighted(leaf_size=4, mode=mode) if mode.uses_primitive_weights() \
        else BvhBuildConfig(mode, 4)
    b = oracle.build_bvh(scene, cfg, bins=bins)
    assert b.node_count == 2 * b.leaf_count - b.root_count
    assert b.ref_count == scene.bounded_primitive_count() and sorted(b.refs.tolist()) == sorted(oracle.build_bvh(scene, cfg).refs.tolist())
    assert _leaf_sizes(b).max() <= 4
    again = oracle.build_bvh(scene, cfg, bins=bins)
    assert again.topology_sha256() == b.topology_sha256()


def test_binned_cost_close_to_full_sweep():
    h = synth.hetero_workload().scene
    full = oracle.build_bvh(h)
    for bins in (16, 32):
        b = oracle.build_bvh(h, bins=bins)
        assert full.generalized_sah <= b.generalized_sah <= 1.02 * full.generalized_sah


def test_binned_median_fallback_keeps_leaf_size():
    m = MaterialData.matte((0.5, 0.5, 0.5))
    s = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 3))
    for _ in range(50):
        s.add_sphere((1.0, 2.0, 3.0), 0.25, m)
    b = oracle.build_bvh(s, bins=8)
    sizes = _leaf_sizes(b)
    assert sizes.max() <= 3 and sizes.sum() == 50
    # the full sweep keeps such a node whole only when no axis has extent (one big leaf)
    assert oracle.build_bvh(s).leaf_count == 1


def test_binned_rejects_bad_bin_counts():
    s = synth.hetero_scene(20, 1, synth.WORKLOAD_IDS["test"], 1)
    for bins in (1, 33):
        with pytest.raises(RuntimeError):
            oracle.build_bvh(s, bins=bins)
