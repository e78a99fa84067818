"""rtb_request_abort on a frame that is running: another host thread raises the context's
abort flag, the persistent render kernel stops fetching work at its next queue fetch, and
the call returns RTB_ERR_WATCHDOG long before the frame would have finished.  Nothing faults
or hangs: the flag is an ordinary device word the kernel polls.  The context stays usable,
and its next frame equals a fresh context's bit for bit."""
import ctypes as C
import threading
import time

import numpy as np
import pytest

from rtb200 import native as N
from rtb200 import synth
from rtb200.tracer import Context, ResidentScene, camera_struct

pytestmark = pytest.mark.gpu


def _params(w, spp, frame):
    return N.RenderParams(w.width, w.height, spp, w.max_depth, frame,
                          w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)


def _frame(ctx, res, w, spp, frame):
    img = np.zeros(w.width * w.height * 3, np.float32)
    cam = camera_struct(w.camera)
    st = ctx.lib.rtb_render_sample(ctx.handle, res.handle, C.byref(cam),
                                   C.byref(_params(w, spp, frame)), N.fptr(img))
    return st, img


def test_abort_request_stops_a_running_frame():
    w = synth.hetero_workload()  # 10k primitives, 1024x1024
    ctx = Context(0)
    try:
        res = ResidentScene.build(ctx, w.scene)
        st, _ = _frame(ctx, res, w, 1, 0)  # warm: kernels loaded, buffers sized
        assert st == N.RTB_OK
        # 1024x1024 at 256 spp is about 268M samples: a second or more on one B200
        timer = threading.Timer(0.15, lambda: ctx.lib.rtb_request_abort(ctx.handle))
        t0 = time.perf_counter()
        timer.start()
        st, _ = _frame(ctx, res, w, 256, 1)
        elapsed = time.perf_counter() - t0
        timer.join()
        assert st == 7, N.STATUS_NAMES.get(st, st)  # RTB_ERR_WATCHDOG
        assert elapsed < 0.8, elapsed
        # the next frame runs to the end and equals the same frame from a fresh context
        st, img = _frame(ctx, res, w, 2, 3)
        assert st == N.RTB_OK
        res.close()
    finally:
        ctx.close()
    ctx2 = Context(0)
    try:
        res2 = ResidentScene.build(ctx2, w.scene)
        st, ref = _frame(ctx2, res2, w, 2, 3)
        assert st == N.RTB_OK
        np.testing.assert_array_equal(img.view(np.int32), ref.view(np.int32))
        res2.close()
    finally:
        ctx2.close()


def test_abort_right_after_async_submits_stops_them_and_spares_later_work():
    """The abort names work by submission: frames submitted with rtb_render_device before
    the call (one running, one still queued behind it) stop at their next work fetch, even
    though the request arrives before either kernel has started reading; a frame submitted
    after the call runs to the end.  Measured by the host clock: the two submitted frames
    would take over a second."""
    torch = pytest.importorskip("torch")
    w = synth.hetero_workload()
    ctx = Context(0)
    try:
        res = ResidentScene.build(ctx, w.scene)
        st, _ = _frame(ctx, res, w, 1, 0)
        assert st == N.RTB_OK
        n = w.width * w.height * 3
        long_out = torch.full((n,), float("nan"), device="cuda")
        queued_out = torch.full((n,), float("nan"), device="cuda")
        later_out = torch.full((n,), float("nan"), device="cuda")
        stream = torch.cuda.Stream()
        torch.cuda.synchronize()
        cam = camera_struct(w.camera)
        sh = C.c_void_p(stream.cuda_stream)
        t0 = time.perf_counter()
        st1 = ctx.lib.rtb_render_device(ctx.handle, res.handle, C.byref(cam),
                                        C.byref(_params(w, 256, 1)),
                                        C.c_void_p(long_out.data_ptr()), sh)
        st2 = ctx.lib.rtb_render_device(ctx.handle, res.handle, C.byref(cam),
                                        C.byref(_params(w, 2, 2)),
                                        C.c_void_p(queued_out.data_ptr()), sh)
        ab = ctx.lib.rtb_request_abort(ctx.handle)
        st3 = ctx.lib.rtb_render_device(ctx.handle, res.handle, C.byref(cam),
                                        C.byref(_params(w, 2, 3)),
                                        C.c_void_p(later_out.data_ptr()), sh)
        stream.synchronize()
        elapsed = time.perf_counter() - t0
        assert (st1, st2, ab, st3) == (N.RTB_OK,) * 4
        assert elapsed < 0.5, elapsed
        # the queued frame saw the abort at its first fetch: nothing was written
        assert torch.isnan(queued_out).all().item()
        # the long frame stopped early: most of it is unwritten
        assert torch.isnan(long_out).float().mean().item() > 0.5
        # the later frame is complete and equals the synchronous render of the same frame
        st, want = _frame(ctx, res, w, 2, 3)
        assert st == N.RTB_OK
        got = later_out.cpu().numpy()
        np.testing.assert_array_equal(got.view(np.int32), want.view(np.int32))
        res.close()
    finally:
        ctx.close()
