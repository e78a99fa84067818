"""Caller-supplied trees that are malformed (rtb_scene_upload with the reference's flattened
BVH arrays, as GpuRayTracer.uploadScene takes them): indices outside the arrays are refused
at upload with RTB_ERR_INVALID_ARGUMENT (ValueError); a cycle back to the root cannot be
seen cheaply at upload, so each ray's node budget (node count + 8) ends its walk and the ray
takes the exhaustive path, which gives exactly the linear-mode hits.  The failures are made
on the host, in the tree arrays; every kernel loop involved is bounded."""
import types

import numpy as np
import pytest

from oracle import oracle
from rtb200 import synth
from rtb200.tracer import GpuRayTracer

pytestmark = pytest.mark.gpu

TYPE_SHIFT = 30


@pytest.fixture(scope="module")
def case():
    scene = synth.hetero_scene(1000, 5, synth.WORKLOAD_IDS["test"], 8)
    rays = synth.primary_grid(synth.camera_looking_z((0.0, 0.0, -2.9)), 32, 18)
    bvh = oracle.build_bvh(scene)
    assert len(bvh.roots) == 1
    return scene, rays, bvh


def _copy(bvh):
    return types.SimpleNamespace(node_bounds=np.array(bvh.node_bounds, copy=True),
                                 node_data=np.array(bvh.node_data, copy=True),
                                 refs=np.array(bvh.refs, copy=True),
                                 roots=np.array(bvh.roots, copy=True),
                                 node_count=bvh.node_count, ref_count=bvh.ref_count,
                                 root_count=bvh.root_count)


def _trace(scene, rays, bvh=None, linear=False, metrics=False):
    with GpuRayTracer(48, 32, 2, not linear) as t:
        return t.trace_replay(scene, rays, collect_metrics=metrics, bvh=bvh)


def _nodes(b):
    return b.node_data.reshape(-1, 4)


def test_reference_index_out_of_range_is_refused(case):
    scene, rays, bvh = case
    bad = _copy(bvh)
    _, counts = scene.arrays()
    per_type = [counts[0], counts[1], counts[3], counts[4]]  # sphere, box, affine sphere, box
    t = int(np.uint32(bad.refs[0]) >> TYPE_SHIFT)
    word = np.array([(t << TYPE_SHIFT) | (per_type[t] + 7)], dtype=np.uint32)
    bad.refs[0] = word.view(np.int32)[0]
    with pytest.raises(ValueError, match="reference index out of range"):
        _trace(scene, rays, bad)


def test_leaf_range_past_the_references_is_refused(case):
    scene, rays, bvh = case
    bad = _copy(bvh)
    nd = _nodes(bad)
    leaf = int(np.nonzero(nd[:, 0] < 0)[0][0])
    nd[leaf, 3] = len(bad.refs) + 5
    with pytest.raises(ValueError, match="out of range"):
        _trace(scene, rays, bad)


def test_child_past_the_nodes_is_refused(case):
    scene, rays, bvh = case
    bad = _copy(bvh)
    nd = _nodes(bad)
    interior = int(np.nonzero(nd[:, 0] >= 0)[0][0])
    nd[interior, 1] = len(nd) + 3
    with pytest.raises(ValueError, match="out of range"):
        _trace(scene, rays, bad)


def test_cycle_back_to_the_root_takes_the_exhaustive_path(case):
    scene, rays, bvh = case
    bad = _copy(bvh)
    nd = _nodes(bad)
    root = int(bad.roots[0])
    interior = [int(i) for i in np.nonzero(nd[:, 0] >= 0)[0] if int(i) != root]
    nd[interior[0], 1] = root  # the right child of a node below the root is the root
    got = _trace(scene, rays, bad, metrics=True)
    want = _trace(scene, rays, linear=True)
    assert got.stats.stack_overflows > 0
    np.testing.assert_array_equal(got.hit_flags, want.hit_flags)
    np.testing.assert_array_equal(got.hit_primitive_orders, want.hit_primitive_orders)
    np.testing.assert_array_equal(got.hit_distances.view(np.int32), want.hit_distances.view(np.int32))


def test_duplicated_reference_traces_the_tree_as_given(case):
    """A reference listed twice (so another primitive is not in the tree): the upload keeps
    the records in their own order instead of renumbering them, and the hits equal the FP32
    restatement's walk of the same tree."""
    scene, rays, bvh = case
    bad = _copy(bvh)
    bad.refs[1] = bad.refs[0]
    got = _trace(scene, rays, bad)
    want = oracle.trace(scene, rays, bad)
    np.testing.assert_array_equal(got.hit_primitive_orders, want["order"])
    np.testing.assert_array_equal(got.hit_distances.view(np.int32), want["t"].view(np.int32))
