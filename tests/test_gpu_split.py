"""rtb_render_rows_device, the unit of a frame split across GPUs, on one device.

For N in 2, 3 and 8 (3 does not divide the height), every rank's interleaved rows (frame rows
r, r + N, ...) are rendered through the C ABI into their own band and assembled with the
split module's reassembly; the frame equals rtb_render_device's full frame bit for bit.
Only one GPU is available here, so the ranks' launches run one after another on it; the
gather between processes is tested with gloo ranks in test_split_ranks.py."""
import ctypes as C

import numpy as np
import pytest

from rtb200 import native as N
from rtb200 import split, synth
from rtb200.tracer import Context, ResidentScene, camera_struct

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3, 8])
def test_interleaved_rows_assemble_to_the_full_frame(world):
    torch = pytest.importorskip("torch")
    w = synth.hetero_workload(width=320, height=181, spp=8, depth=6)
    ctx = Context(0)
    try:
        res = ResidentScene.build(ctx, w.scene)
        p = N.RenderParams(w.width, w.height, w.spp, w.max_depth, 5,
                           w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
        cam = camera_struct(w.camera)
        full = torch.empty(w.width * w.height * 3, device="cuda")
        ctx.check(ctx.lib.rtb_render_device(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                            C.c_void_p(full.data_ptr()), None))
        k = split.band_rows(w.height, world)
        gathered = torch.full((world * k * w.width * 3,), float("nan"), device="cuda")
        render_rows = split.device_rows_renderer(ctx, res, cam, p)
        for r in range(world):
            render_rows(r, world, gathered[r * k * w.width * 3:(r + 1) * k * w.width * 3])
        torch.cuda.synchronize()
        img = split.assemble(gathered, w.height, w.width, world)
        a = img.contiguous().cpu().numpy().reshape(-1)
        b = full.cpu().numpy()
        np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))
        # a first row outside the frame is refused
        st = ctx.lib.rtb_render_rows_device(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                            w.height, world, C.c_void_p(full.data_ptr()), None)
        assert st == 1  # RTB_ERR_INVALID_ARGUMENT
        res.close()
    finally:
        ctx.close()
