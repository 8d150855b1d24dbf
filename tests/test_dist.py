"""Multi-process plumbing of bench.py on CPU (gloo, world size 2): the timed
interval is the maximum over ranks, every rank takes the same collective steps
(barrier, all-reduce), and the whole-job value counts every rank's cells.
Replicas only: the engine path has no data-path collective."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        elapsed = 1.0 + rank  # rank 1 is the slow one
        t = bench.max_over_ranks(elapsed, world, torch.device("cpu"))
        cells, steps = 1000, 10
        value = cells * steps * world / t / 1e9
        bench.barrier(world)
        out.put((rank, t, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[0] for r in res] == [0, 1]
    for _, t, value in res:
        assert t == pytest.approx(2.0)  # the slower rank's interval on every rank
        assert value == pytest.approx(1000 * 10 * 2 / 2.0 / 1e9)
