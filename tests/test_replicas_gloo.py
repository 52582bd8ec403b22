"""The multi-rank path of bench.py (replicas: one independent solve per rank,
no data-path collective) on CPU with two gloo ranks: the max over ranks that
sets the job's time, and the reference arm's rank-0-only rule."""
from __future__ import annotations

import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r reports (10 + r, 100 - r): the job's time is the slowest rank's on each entry
        got = bench.max_over_ranks([10.0 + rank, 100.0 - rank], dist)
        dist.barrier()
        # ranks other than 0 leave the reference arm at once, without output
        quiet = bench.reference_arm(None, rank, world) if rank != 0 else None
        q.put((rank, got, quiet))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, got, quiet in res:
        assert got == [11.0, 100.0]
        assert quiet is None


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([3.0, 4.5]) == [3.0, 4.5]
