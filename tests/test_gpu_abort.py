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
