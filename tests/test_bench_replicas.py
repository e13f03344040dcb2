"""bench.py with N GPUs runs N independent replicas: the job's time is the slowest rank's and its
edge count is the sum over ranks.  Checked with two gloo ranks on CPU."""
from __future__ import annotations

import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import os

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms, edges = bench.replica_totals(10.0 * (rank + 1), 1000 + rank, world, device="cpu")
        out.put((rank, ms, edges))
    finally:
        dist.destroy_process_group()


def test_replica_totals_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for _, ms, edges in got:
        assert ms == 20.0 and edges == 2001


def test_replica_totals_one_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.replica_totals(12.5, 77, 1) == (12.5, 77)
