"""One frame split over ranks (rtb200.split), on CPU with gloo ranks.

Each rank renders its interleaved rows (frame rows r, r + N, ...) with the FP32 restatement
of the kernel standing in for rtb_render_rows_device (same pixel-keyed random streams), the
bands are all-gathered, and the assembled frame must equal a single-process render of the
whole frame bit for bit: the gather and the reassembly move bytes only.  World sizes 2 and 3
(3 does not divide the height, so the last bands are padded).  The GPU side of the same split
(every rank's rows rendered on one device and assembled) is tested in test_gpu_split.py."""
import dataclasses
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    from rtb200 import synth
    base = synth.plain_workload()
    return dataclasses.replace(base, width=10, height=7, spp=2, max_depth=3, frame_index=4,
                               camera=synth.camera_looking_z(base.camera.position, 10 / 7))


def _rank_main(rank, world, port, outdir):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        sys.path.insert(0, ROOT)
        sys.path.insert(0, os.path.join(ROOT, "master-rad_b200"))
        import datetime

        from oracle import oracle
        from rtb200 import split
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        w = _workload()

        def render_rows(first_row, row_stride, band):
            rows = range(first_row, w.height, row_stride)
            for k, y in enumerate(rows):
                img = oracle.render(w, pixel_begin=y * w.width, pixel_end=(y + 1) * w.width)
                band[k * w.width * 3:(k + 1) * w.width * 3] = torch.from_numpy(img.reshape(-1))

        frame = split.render_split_frame(render_rows, torch, w.height, w.width, world, rank)
        np.save(os.path.join(outdir, "frame%d.npy" % rank), frame.numpy())
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:  # noqa: BLE001 - reported to the parent
        import traceback
        with open(os.path.join(outdir, "err%d" % rank), "w") as f:
            f.write("".join(traceback.format_exception(e)))
        raise


@pytest.mark.parametrize("world", [2, 3])
def test_split_frame_over_gloo_ranks_equals_single_render(tmp_path, world):
    try:
        mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                           join=True, start_method="spawn")
    except Exception:
        msgs = [open(tmp_path / ("err%d" % r)).read() for r in range(world)
                if (tmp_path / ("err%d" % r)).exists()]
        pytest.fail("\n".join(msgs) or "rank failed")
    sys.path.insert(0, ROOT)
    from oracle import oracle
    w = _workload()
    want = oracle.render(w).reshape(w.height, w.width, 3)
    for r in range(world):
        got = np.load(tmp_path / ("frame%d.npy" % r))
        np.testing.assert_array_equal(got.view(np.int32), want.view(np.int32))


def test_band_arithmetic():
    from rtb200 import split
    for h in (1, 7, 1024, 1080):
        for n in (1, 2, 3, 4, 8):
            k = split.band_rows(h, n)
            assert sum(split.rows_of_rank(h, n, r) for r in range(n)) == h
            assert all(split.rows_of_rank(h, n, r) <= k for r in range(n))
            g = torch.arange(n * k * 2 * 3, dtype=torch.float32)
            img = split.assemble(g, h, 2, n)
            # frame row y is rank y % n's band row y // n
            for y in (0, h - 1, h // 2):
                r, kk = y % n, y // n
                want = g.view(n, k, 2, 3)[r, kk]
                assert torch.equal(img[y], want)
