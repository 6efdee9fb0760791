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


def _slice_main(rank, world, port, out):
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = torch.tensor(bench.rank_columns(rank, world, 55296), dtype=torch.int64)
        every = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(every, mine)
        out.put((rank, [tuple(t.tolist()) for t in every]))
    finally:
        dist.destroy_process_group()


def test_rank_slices_partition_the_domain():
    """Each rank's columns, gathered over two gloo ranks, tile the job's
    domain exactly once: no column is shared and none is left out."""
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slice_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slices in res:
        assert slices == [(0, 55296), (55296, 110592)]
        covered = sorted(c for a, b in slices for c in range(a, b))
        assert covered == list(range(world * 55296))


def test_gpus_flag_launches_its_ranks():
    """``bench.py --gpus 2`` from a single process starts two ranks itself
    (torch.distributed.run); on the reference arm rank 0 alone prints the
    line. A tiny C2 domain keeps the oracle's work to a fraction of a second."""
    import json
    import subprocess

    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3", "--ncube", "2"], capture_output=True, text=True, env=env,
                       timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    rec = lines[0]
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["steps"] == 1
    assert rec["config"]["columns_per_gpu"] == 24 and rec["value"] > 0
