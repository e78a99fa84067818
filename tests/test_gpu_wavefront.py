"""rtb_render_device_wavefront, the wavefront form of a frame (one wave per sample index,
per bounce a trace kernel over the live paths and a shade kernel), against the persistent
kernel behind rtb_render_device: the same frames bit for bit, on the plain and the
heterogeneous scene (every primitive type, mixed leaves), a frame too deep for any path to
end early, depth 0 (black samples) and one sample per pixel; the metrics build is refused."""
import ctypes as C

import numpy as np
import pytest

from rtb200 import native as N
from rtb200 import synth
from rtb200.tracer import Context, ResidentScene, camera_struct

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _frames(ctx, w, spp, depth, metrics=0):
    torch = pytest.importorskip("torch")
    res = ResidentScene.build(ctx, w.scene)
    try:
        p = N.RenderParams(w.width, w.height, spp, depth, 3, w.frame_seed & 0xFFFFFFFFFFFFFFFF,
                           1, metrics, 0)
        cam = camera_struct(w.camera)
        out = []
        for fn in (ctx.lib.rtb_render_device, ctx.lib.rtb_render_device_wavefront):
            img = torch.full((w.width * w.height * 3,), float("nan"), device="cuda")
            st = fn(ctx.handle, res.handle, C.byref(cam), C.byref(p), C.c_void_p(img.data_ptr()),
                    None)
            torch.cuda.synchronize()
            out.append((st, img.cpu().numpy()))
        return out
    finally:
        res.close()


@pytest.mark.parametrize("kind,spp,depth", [("plain", 8, 4), ("hetero", 4, 8), ("hetero", 1, 32),
                                            ("hetero", 3, 0), ("plain", 1, 1)])
def test_wavefront_frame_equals_the_persistent_kernel(ctx, kind, spp, depth):
    w = (synth.plain_workload() if kind == "plain"
         else synth.hetero_workload(width=200, height=150, spp=spp, depth=depth))
    (s0, a), (s1, b) = _frames(ctx, w, spp, depth)
    assert s0 == 0 and s1 == 0
    assert np.isfinite(b).all()
    np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))


@pytest.mark.parametrize("width,height", [(1, 1), (7, 3), (33, 5)])
def test_wavefront_odd_frame_sizes(ctx, width, height):
    """Frames smaller than a warp or a block, and sizes that are not multiples of either."""
    w = synth.hetero_workload(width=width, height=height, spp=5, depth=6)
    (s0, a), (s1, b) = _frames(ctx, w, 5, 6)
    assert s0 == 0 and s1 == 0
    np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))


def test_wavefront_refuses_the_metrics_build(ctx):
    w = synth.plain_workload()
    (_, _), (st, _) = _frames(ctx, w, 1, 2, metrics=1)
    assert st == 5  # RTB_ERR_UNSUPPORTED
