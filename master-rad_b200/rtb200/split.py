"""One frame rendered by N processes, one per GPU, and gathered.

The reference renders a frame on one device (gfxlab/gpu/GpuRayTracer.java:796 binds one
context; its tile plan, gfxlab/gpu/GpuLaunchProvenance.java:44-60, splits a frame into
launches on that device).  Here the frame's rows are dealt out across ranks: rank r of N
renders frame rows r, r + N, r + 2N, ... with ``rtb_render_rows_device`` into a band of
ceil(H / N) rows (the last ones unused where N does not divide H), and one all-gather over
NCCL (NVLink / NVSwitch) brings every band to every rank, where the rows are put back in
frame order.  Interleaved rows balance the uneven cost of image regions (a band of
consecutive rows that holds the emitter or most of the geometry would set the pace).

Every pixel's random streams are keyed by its frame pixel index, so the gathered frame
equals the single-GPU frame bit for bit; the gather moves bytes only.
"""
from __future__ import annotations

import ctypes as C


def band_rows(height: int, world: int) -> int:
    """Rows in every rank's band (the gather needs equal sizes)."""
    return -(-height // world)


def rows_of_rank(height: int, world: int, rank: int) -> int:
    """Frame rows rank `rank` renders: rank, rank + world, ... below height."""
    return len(range(rank, height, world))


def assemble(gathered, height: int, width: int, world: int):
    """Frame-order image (height x width x 3) from the all-gathered bands, which hold rank
    r's row k (frame row r + k * world) at [r, k]."""
    k = band_rows(height, world)
    return gathered.view(world, k, width, 3).transpose(0, 1).reshape(k * world, width, 3)[:height]


def render_split_frame(render_rows, torch, height: int, width: int, world: int, rank: int,
                       group=None, band=None, gathered=None):
    """Renders this rank's rows with ``render_rows(first_row, row_stride, band_tensor)`` and
    all-gathers the bands; returns the whole frame (height x width x 3) on every rank.
    ``band`` and ``gathered`` may be passed to reuse buffers (sizes: band_rows x width x 3
    and world times that)."""
    import torch.distributed as dist
    k = band_rows(height, world)
    if band is None:
        dev = "cuda" if torch.cuda.is_available() and dist.get_backend(group) == "nccl" else "cpu"
        band = torch.zeros(k * width * 3, dtype=torch.float32, device=dev)
    if gathered is None:
        gathered = torch.empty(world * band.numel(), dtype=band.dtype, device=band.device)
    if rows_of_rank(height, world, rank) > 0:
        render_rows(rank, world, band)
    dist.all_gather_into_tensor(gathered, band, group=group)
    return assemble(gathered, height, width, world)


def device_rows_renderer(ctx, resident, camera_struct, params, stream=None):
    """The product renderer for render_split_frame: rtb_render_rows_device into the band's
    device memory on ``stream`` (a cudaStream_t handle; None: the context's stream)."""

    def render_rows(first_row, row_stride, band):
        ctx.check(ctx.lib.rtb_render_rows_device(ctx.handle, resident.handle, C.byref(camera_struct),
                                                 C.byref(params), first_row, row_stride,
                                                 C.c_void_p(band.data_ptr()),
                                                 C.c_void_p(stream) if stream else None))

    return render_rows
