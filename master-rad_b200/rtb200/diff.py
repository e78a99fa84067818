"""Differentiable rendering: per-material albedo and emission as torch parameters.

``RenderFunction`` is the forward/backward Function of the path tracer (the Java analogue is
a Function object with forward and backward methods over the same C ABI): forward writes the
parameters into the resident scene's material records and renders the frame; backward runs
the path-replay adjoint (rtb_render_backward) on the incoming image gradient and returns
dLoss/d(albedo) and dLoss/d(emission), one RGB triple per material record.  Materials are
deduplicated by value as the reference's GpuScene does, so in scenes whose primitives have
distinct colours these are per-primitive gradients.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .tracer import Context, ResidentScene, camera_struct


class DifferentiableScene:
    def __init__(self, ctx: Context, scene, width: int, height: int, spp: int, max_depth: int,
                 camera, frame_index: int = 0, frame_seed: int = 1):
        self.ctx = ctx
        self.res = ResidentScene.build(ctx, scene)
        self.base = scene.material_data().reshape(-1, 13).copy()
        self.count = len(self.base)
        self.params = N.RenderParams(width, height, spp, max_depth, frame_index,
                                     int(frame_seed) & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
        self.cam = camera_struct(camera)
        self.width, self.height = width, height

    def albedo(self) -> np.ndarray:
        return self.base[:, 0:3].copy()

    def emission(self) -> np.ndarray:
        return self.base[:, 9:12].copy()

    def set_parameters(self, albedo, emission) -> None:
        m = self.base.copy()
        m[:, 0:3] = np.asarray(albedo, dtype=np.float32).reshape(-1, 3)
        m[:, 9:12] = np.asarray(emission, dtype=np.float32).reshape(-1, 3)
        m = np.ascontiguousarray(m, dtype=np.float32)
        self.ctx.check(self.ctx.lib.rtb_scene_set_materials(self.ctx.handle, self.res.handle,
                                                            N.fptr(m.reshape(-1)), self.count))

    def render_into(self, out_ptr: int, stream=None) -> None:
        self.ctx.check(self.ctx.lib.rtb_render_device(self.ctx.handle, self.res.handle,
                                                      C.byref(self.cam), C.byref(self.params),
                                                      C.c_void_p(out_ptr),
                                                      C.c_void_p(stream) if stream else None))

    def backward_into(self, adjoint_ptr: int, grad_albedo_ptr: int, grad_emission_ptr: int,
                      stream=None) -> None:
        self.ctx.check(self.ctx.lib.rtb_render_backward(
            self.ctx.handle, self.res.handle, C.byref(self.cam), C.byref(self.params),
            C.c_void_p(adjoint_ptr), C.c_void_p(grad_albedo_ptr), C.c_void_p(grad_emission_ptr),
            C.c_void_p(stream) if stream else None))

    def close(self):
        self.res.close()


def torch_stream_handle(torch) -> int:
    """The current torch stream as a cudaStream_t for the C ABI.  torch's legacy default
    stream has handle 0, which the C ABI reads as "the context's own stream"; pass
    cudaStreamLegacy (1) instead so the launch orders with torch's work."""
    h = torch.cuda.current_stream().cuda_stream
    return h if h else 1


def render_function():
    """The torch.autograd.Function (built lazily so that importing this module does not
    require torch)."""
    import torch

    class RenderFunction(torch.autograd.Function):
        @staticmethod
        def forward(fctx, albedo, emission, dscene):
            dscene.set_parameters(albedo.detach().cpu().numpy(), emission.detach().cpu().numpy())
            img = torch.empty(dscene.width * dscene.height * 3, dtype=torch.float32, device="cuda")
            dscene.render_into(img.data_ptr(), torch_stream_handle(torch))
            fctx.dscene = dscene
            fctx.devices = (albedo.device, emission.device)
            return img

        @staticmethod
        def backward(fctx, grad_image):
            d = fctx.dscene
            g = grad_image.detach().to(device="cuda", dtype=torch.float32).contiguous()
            ga = torch.empty(d.count * 3, dtype=torch.float32, device="cuda")
            ge = torch.empty(d.count * 3, dtype=torch.float32, device="cuda")
            d.backward_into(g.data_ptr(), ga.data_ptr(), ge.data_ptr(), torch_stream_handle(torch))
            return (ga.view(d.count, 3).to(fctx.devices[0]), ge.view(d.count, 3).to(fctx.devices[1]),
                    None)

    return RenderFunction
