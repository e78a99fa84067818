"""Helpers of bench.py: the two roofline bounds it reports for the render launch
(algorithmic bytes against the HBM copy bandwidth, and warp instructions against the SMs'
issue rate, one instruction per cycle on each of an SM's 4 schedulers), and how the batched
workload's scenes are dealt to ranks."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "master-rad_b200"))

import bench  # noqa: E402


def test_issue_roofline_arithmetic():
    samples = 1024 * 1024 * 64
    r = bench.issue_roofline("hetero", samples, 250.0, 148, 2000.0)
    inst = bench.INST_PER_SAMPLE["hetero"] * samples
    assert r["bound"] == "issue" and r["unit"] == "warp-inst/s"
    assert r["inst_per_launch"] == pytest.approx(inst)
    assert r["achieved"] == pytest.approx(inst / 0.25)
    assert r["peak"] == pytest.approx(148 * 4 * 2000e6)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])


def test_issue_roofline_needs_a_capture_and_a_clock():
    assert bench.issue_roofline("plain", 100, 1.0, 148, 1965.0) is None
    assert bench.issue_roofline("hetero", 100, 1.0, 148, None) is None


def test_algorithmic_bytes_formula():
    # rays, aabb, prim, sphere, box, plane, aff-sphere, aff-box, ovf, max, internal, leaf, h, m
    c = (10, 0, 0, 3, 2, 6, 1, 1, 0, 0, 5, 0, 0, 0)
    want = 64 * 5 + 16 * 3 + 32 * 2 + 48 * 2 + 4 * 7 + 16 * 6 + 100 * 4
    assert bench.algorithmic_bytes(c, 4) == want


@pytest.fixture(scope="module")
def batched_works():
    from rtb200 import synth
    return synth.batched_workloads()


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_batched_scenes_are_dealt_to_ranks_without_overlap(world, batched_works):
    """--workload batched under N ranks: every one of the 64 scenes is rendered by exactly one
    rank, so the job's samples are the sum of the ranks' shares."""
    works = batched_works
    shares = [bench.scenes_of_rank(len(works), r, world) for r in range(world)]
    flat = sorted(i for sh in shares for i in sh)
    assert flat == list(range(len(works)))
    total = sum(w.width * w.height * w.spp for w in works)
    assert sum(works[i].width * works[i].height * works[i].spp
               for sh in shares for i in sh) == total
    assert max(len(sh) for sh in shares) - min(len(sh) for sh in shares) <= 1
