"""Batched rendering over the C ABI: many resident scenes in one persistent launch replayed
from a CUDA graph (rtb_batch_* in include/rtb200.h), with the autotuner's choice of launch
parameters cached per device and batch shape."""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import List, Optional, Sequence

from . import native as N
from .tracer import Context, ResidentScene, camera_struct


class Batch:
    """jobs: (ResidentScene, GpuCamera, width, height, spp, max_depth, frame_index, frame_seed,
    output device pointer) tuples; outputs are caller-owned device buffers of 3 floats per
    pixel (for example torch CUDA tensors)."""

    def __init__(self, ctx: Context, jobs: Sequence[tuple], tuning: Optional[dict] = None):
        self.ctx = ctx
        arr = (N.BatchJob * len(jobs))()
        self._keep = []
        for k, (res, cam, w, h, spp, depth, frame_index, frame_seed, out_ptr) in enumerate(jobs):
            arr[k].scene = res.handle.value if isinstance(res.handle, C.c_void_p) else res.handle
            arr[k].camera = camera_struct(cam)
            arr[k].params = N.RenderParams(w, h, spp, depth, frame_index,
                                           int(frame_seed) & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
            arr[k].rgb_device = out_ptr
        self._jobs = arr
        t = None
        if tuning is not None:
            t = N.BatchTuning(int(tuning["threads_per_block"]), int(tuning["job_order"]),
                              int(tuning.get("branches", 0)),
                              int(tuning.get("shared_stack_entries", 0)),
                              int(tuning.get("tail_pixels_per_thread", 0)))
        h = C.c_void_p()
        ctx.check(ctx.lib.rtb_batch_create(ctx.handle, arr, len(jobs), C.byref(t) if t else None,
                                           C.byref(h)))
        self.handle = h

    def render(self, stream=None):
        self.ctx.check(self.ctx.lib.rtb_batch_render(self.ctx.handle, self.handle,
                                                     C.c_void_p(stream) if stream else None))

    def autotune(self, repeats: int = 2) -> dict:
        best = N.BatchTuning()
        ms = C.c_double()
        self.ctx.check(self.ctx.lib.rtb_batch_autotune(self.ctx.handle, self.handle, repeats,
                                                       C.byref(best), C.byref(ms)))
        return {"threads_per_block": best.threads_per_block, "job_order": best.job_order,
                "branches": best.branches, "shared_stack_entries": best.shared_stack_entries,
                "tail_pixels_per_thread": best.tail_pixels_per_thread, "ms": ms.value}

    def close(self):
        if self.handle:
            self.ctx.lib.rtb_batch_destroy(self.ctx.handle, self.handle)
            self.handle = None


def tuning_cache_path() -> str:
    return os.environ.get("RTB_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "rtb200_tuning.json"))


def cached_tuning(key: str) -> Optional[dict]:
    try:
        with open(tuning_cache_path()) as f:
            return json.load(f).get(key)
    except (OSError, ValueError):
        return None


def store_tuning(key: str, value: dict) -> None:
    path = tuning_cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = {}
        if os.path.exists(path):
            with open(path) as f:
                data = json.load(f)
        data[key] = value
        with open(path, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    except (OSError, ValueError):
        pass


def batch_key(device_name: str, jobs: Sequence[tuple]) -> str:
    """(device, configuration class): job count and the spread of frame costs."""
    costs = sorted(int(j[2]) * int(j[3]) * int(j[4]) * max(1, int(j[5])) for j in jobs)
    return "%s|jobs=%d|cost_min=%d|cost_max=%d" % (device_name, len(jobs), costs[0], costs[-1])
