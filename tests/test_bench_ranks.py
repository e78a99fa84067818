"""The N > 1 path of bench.py on CPU: two gloo ranks take the bench's own rank logic
(disjoint frame ranges per rank, max-over-ranks timing, whole-job rate, rank-0-only
reference arm) and render their first frames with the FP32 restatement of the kernel, so the
frames each rank contributes are shown to be distinct work."""
import dataclasses
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, errfile):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                          WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
        sys.path.insert(0, ROOT)
        import datetime

        import bench
        from oracle import oracle
        from rtb200 import synth
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))

        # max over ranks of each rank's timed milliseconds, as the bench reduces them
        ms = 10.0 + 5.0 * rank
        slowest = bench.max_over_ranks(ms, device="cpu")
        assert slowest == 10.0 + 5.0 * (world - 1), slowest
        rate = bench.whole_job_rate(world, 4, 1000, slowest / 1e3)
        assert abs(rate - world * 4 * 1000 / (slowest / 1e3) / 1e6) < 1e-12

        # the frames every rank touches (counters, warm-up, timed, end-to-end) are disjoint
        steps, warmup = 8, 3
        mine = {bench.frame_index(rank, 0)}
        mine |= {bench.frame_index(rank, i, 1000) for i in range(warmup)}
        mine |= {bench.frame_index(rank, i) for i in range(steps)}
        mine |= {bench.frame_index(rank, i, 500) for i in range(warmup + steps)}
        every = [None] * world
        dist.all_gather_object(every, sorted(mine))
        for a in range(world):
            for b in range(a + 1, world):
                assert not set(every[a]) & set(every[b]), (a, b)

        # each rank's first timed frame is different work; the same frame is reproducible
        base = synth.plain_workload()
        w = dataclasses.replace(base, width=12, height=12, spp=2, max_depth=3,
                                frame_index=bench.frame_index(rank, 0))
        img = oracle.render(w)
        assert np.array_equal(img, oracle.render(w))
        imgs = [None] * world
        dist.all_gather_object(imgs, img)
        for a in range(world):
            for b in range(a + 1, world):
                assert not np.array_equal(imgs[a], imgs[b])

        # the reference arm prints from rank 0 only; other ranks leave without work
        if rank != 0:
            args = bench.parse_args(["--impl", "reference", "--gpus", str(world)])
            buf = io.StringIO()
            with redirect_stdout(buf):
                bench.run_reference(args)
            assert buf.getvalue() == ""
        dist.barrier()
        dist.destroy_process_group()
    except BaseException as e:  # noqa: BLE001 - reported to the parent
        import traceback
        with open(errfile + ".%d" % rank, "w") as f:
            f.write("".join(traceback.format_exception(e)))
        raise


def test_two_gloo_ranks_follow_the_bench_rank_logic(tmp_path):
    world = 2
    err = str(tmp_path / "err")
    try:
        mp.start_processes(_rank_main, args=(world, _free_port(), err), nprocs=world,
                           join=True, start_method="spawn")
    except Exception:
        msgs = [open(err + ".%d" % r).read() for r in range(world)
                if os.path.exists(err + ".%d" % r)]
        pytest.fail("\n".join(msgs) or "rank failed")
