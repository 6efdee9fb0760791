"""Multi-rank host logic of bench.py, on CPU with the gloo backend.

Every column is independent, so N GPUs run N replicas (one per rank) with no
collective on the data path; the only exchange is the max over ranks of the
device-measured times, from which rank 0 derives the whole-job rate. These
tests run that logic in two real processes over gloo.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # rank r "measured" these times (ms): the total, e2e, per-launch mean
        mine = [100.0 + 10.0 * rank, 50.0 - rank, 4.0 + rank]
        got = bench.max_over_ranks(mine, world, torch.device("cpu"))
        rate = bench.whole_job_rate(world, 55296, 10, got[0])
        dist.barrier()
        out.put((rank, got, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_two_ranks():
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, rate in res:
        # the slowest replica's times on every rank
        assert got == [110.0, 50.0, 5.0]
        # 2 replicas x 55,296 columns x 10 steps in 110 ms
        assert rate == pytest.approx(2 * 55296 * 10 / 0.110, rel=1e-15)


def test_single_rank_needs_no_process_group():
    import torch

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3.0, 1.0], 1, torch.device("cpu")) == [3.0, 1.0]
    assert bench.whole_job_rate(1, 864, 2, 1000.0) == 1728.0
