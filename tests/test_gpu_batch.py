"""Batched rendering: one persistent launch over several scenes of uneven size, resolution,
sample count and depth (replayed from a CUDA graph) gives every scene exactly the image of
its own frame."""
import ctypes as C

import numpy as np
import pytest

from rtb200 import native as N
from rtb200 import synth
from rtb200.batch import Batch
from rtb200.tracer import Context, ResidentScene, camera_struct

pytestmark = pytest.mark.gpu


def _single(ctx, res, w, torch):
    out = torch.zeros(w.width * w.height * 3, dtype=torch.float32, device="cuda")
    p = N.RenderParams(w.width, w.height, w.spp, w.max_depth, w.frame_index, w.frame_seed, 1, 0, 0)
    cam = camera_struct(w.camera)
    ctx.check(ctx.lib.rtb_render_device(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                        C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_batch_matches_per_scene_frames():
    torch = pytest.importorskip("torch")
    ctx = Context(0)
    try:
        specs = [(1200, 64, 48, 4, 3), (300, 96, 96, 2, 6), (5000, 40, 72, 3, 4), (50, 17, 9, 5, 2),
                 (2000, 128, 64, 1, 8)]
        works, outs, jobs = [], [], []
        for i, (n, wdt, hgt, spp, depth) in enumerate(specs):
            s = synth.hetero_scene(n, 300 + i, synth.WORKLOAD_IDS["test"], 20 + i)
            w = synth.Workload("b%d" % i, s, synth.camera_looking_z((0.0, 0.0, -2.9), wdt / hgt),
                               wdt, hgt, spp, depth, frame_seed=1000 + 7 * i, frame_index=i)
            res = ResidentScene.build(ctx, s)
            out = torch.zeros(wdt * hgt * 3, dtype=torch.float32, device="cuda")
            works.append((w, res))
            outs.append(out)
            jobs.append((res, w.camera, wdt, hgt, spp, depth, w.frame_index, w.frame_seed, out.data_ptr()))
        b = Batch(ctx, jobs)
        for _ in range(2):  # graph replay twice
            for o in outs:
                o.zero_()
            b.render()
            torch.cuda.synchronize()
            for (w, res), o in zip(works, outs):
                np.testing.assert_array_equal(o.cpu().numpy().view(np.int32),
                                              _single(ctx, res, w, torch).view(np.int32))
        best = b.autotune(repeats=1)
        assert best["threads_per_block"] in (64, 128, 256) and best["job_order"] in (0, 1)
        assert best["branches"] in (0, 1, 2, 4)
        for o in outs:
            o.zero_()
        b.render()
        torch.cuda.synchronize()
        for (w, res), o in zip(works, outs):
            np.testing.assert_array_equal(o.cpu().numpy().view(np.int32),
                                          _single(ctx, res, w, torch).view(np.int32))
        b.close()
        for _, res in works:
            res.close()
    finally:
        ctx.close()


def test_batch_tail_spanning_jobs():
    """A batch larger than two pixels per resident thread: in the shared-queue kernel the
    first job runs whole pixels and the single-sample tail covers the last job and part of
    the one before it; in frames mode (1, 2 or 4 graph branches) each job is its own frame
    with its own queue and sample buffer."""
    torch = pytest.importorskip("torch")
    ctx = Context(0)
    try:
        specs = [(800, 512, 384, 2, 3), (400, 512, 384, 3, 3), (600, 512, 384, 1, 4)]
        works, outs, jobs = [], [], []
        for i, (n, wdt, hgt, spp, depth) in enumerate(specs):
            s = synth.hetero_scene(n, 500 + i, synth.WORKLOAD_IDS["test"], 30 + i)
            w = synth.Workload("t%d" % i, s, synth.camera_looking_z((0.0, 0.0, -2.9), wdt / hgt),
                               wdt, hgt, spp, depth, frame_seed=77 + i, frame_index=i)
            res = ResidentScene.build(ctx, s)
            out = torch.zeros(wdt * hgt * 3, dtype=torch.float32, device="cuda")
            works.append((w, res))
            outs.append(out)
            jobs.append((res, w.camera, wdt, hgt, spp, depth, w.frame_index, w.frame_seed, out.data_ptr()))
        tunings = [{"threads_per_block": 128, "job_order": o, "branches": k}
                   for o in (0, 1) for k in (0, 1, 2, 4)]
        # the autotuner's other knobs: end-of-frame queue granularity and shared-memory
        # stack depth change the schedule, never the images
        tunings += [{"threads_per_block": 128, "job_order": 1, "branches": 2,
                     "shared_stack_entries": se, "tail_pixels_per_thread": tp}
                    for se, tp in ((-1, 1), (8, 8), (16, 2))]
        tunings += [{"threads_per_block": 64, "job_order": 0, "branches": 0,
                     "tail_pixels_per_thread": tp} for tp in (1, 8)]
        for tuning in tunings:
            b = Batch(ctx, jobs, tuning=tuning)
            b.render()
            torch.cuda.synchronize()
            for (w, res), o in zip(works, outs):
                np.testing.assert_array_equal(o.cpu().numpy().view(np.int32),
                                              _single(ctx, res, w, torch).view(np.int32))
                o.zero_()
            b.close()
        for _, res in works:
            res.close()
    finally:
        ctx.close()


def test_batch_mixes_tree_and_linear_scenes():
    """The shared-queue kernel with a scene that has a tree beside one that has none (tested
    primitive by primitive): warps at the boundary hold lanes of both, and every image still
    equals its own frame."""
    torch = pytest.importorskip("torch")
    ctx = Context(0)
    try:
        works, outs, jobs, scenes = [], [], [], []
        for i, (n, tree) in enumerate([(300, True), (120, False), (500, True)]):
            s = synth.hetero_scene(n, 700 + i, synth.WORKLOAD_IDS["test"], 40 + i)
            w = synth.Workload("m%d" % i, s, synth.camera_looking_z((0.0, 0.0, -2.9), 40 / 30),
                               40, 30, 3, 4, frame_seed=300 + i, frame_index=i)
            res = ResidentScene.build(ctx, s) if tree else ResidentScene.upload(ctx, s, None)
            out = torch.zeros(40 * 30 * 3, dtype=torch.float32, device="cuda")
            works.append((w, res))
            outs.append(out)
            jobs.append((res, w.camera, 40, 30, 3, 4, w.frame_index, w.frame_seed, out.data_ptr()))
        for threads in (64, 128, 256):
            b = Batch(ctx, jobs, tuning={"threads_per_block": threads, "job_order": 0, "branches": 0})
            b.render()
            torch.cuda.synchronize()
            for (w, res), o in zip(works, outs):
                np.testing.assert_array_equal(o.cpu().numpy().view(np.int32),
                                              _single(ctx, res, w, torch).view(np.int32))
                o.zero_()
            b.close()
        for _, res in works:
            res.close()
    finally:
        ctx.close()


def test_batch_rejects_bad_tuning_knobs():
    torch = pytest.importorskip("torch")
    ctx = Context(0)
    try:
        s = synth.hetero_scene(50, 901, synth.WORKLOAD_IDS["test"], 50)
        res = ResidentScene.build(ctx, s)
        out = torch.zeros(8 * 8 * 3, device="cuda")
        cam = synth.camera_looking_z((0.0, 0.0, -2.9))
        jobs = [(res, cam, 8, 8, 1, 2, 0, 1, out.data_ptr())]
        from rtb200 import native as N
        for bad in ({"shared_stack_entries": 4}, {"tail_pixels_per_thread": 17}):
            t = {"threads_per_block": 128, "job_order": 0, "branches": 1}
            t.update(bad)
            with pytest.raises(ValueError):
                Batch(ctx, jobs, tuning=t)
        res.close()
    finally:
        ctx.close()
