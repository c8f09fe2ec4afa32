"""The multi-rank path of bench.py on CPU: two gloo ranks, as torchrun would
launch them (one instance per rank, no data-path collective).  The timing
reduction takes the slowest rank, the job rate counts every rank's units
over that time, and the reference arm runs on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as tdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench
        times = bench.max_over_ranks([1.0 + rank, 5.0 - rank, 0.25 * rank], world, "cpu")

        class Args:
            steps, warmup, nx = 2, 3, 128
        buf = io.StringIO()
        if rank != 0:
            with redirect_stdout(buf):
                bench.run_reference(Args(), rank, world)
        out[rank] = (times, buf.getvalue())
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank_and_rank0_reports():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        times, printed = res[r]
        assert times == [2.0, 5.0, 0.25], (r, times)
    assert res[1][1] == ""  # the reference arm prints nothing on other ranks


def test_job_rate_counts_all_ranks_over_the_slowest():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_rate(4, 1e6, 2.0) == pytest.approx(2e6)
    assert bench.job_rate(1, 3e6, 1.5) == pytest.approx(2e6)
