"""bench.py's multi-rank bookkeeping on CPU: two gloo ranks, the slowest
rank's time, and the whole-job rate of weak scaling."""

from __future__ import annotations

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu")
        rate = bench.whole_job_rate(1000, 4, slowest, world)
        q.put((rank, slowest, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, slowest, rate in got:
        assert slowest == 15.0  # rank 1's 15 ms
        assert rate == pytest.approx(2 * 1000 * 4 / 0.015)


def test_single_process_is_its_own_max():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, "cpu") == 3.5
    assert bench.whole_job_rate(10, 2, 1000.0, 1) == pytest.approx(20.0)
