"""The multi-GPU path is replicas only: every rank runs its own packing and
the only exchange is the max of the per-rank timings (bench.py). This checks
that host logic with two gloo ranks on the CPU."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as tmp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r, w, lr = bench.dist_env()
    assert (r, w, lr) == (rank, world, rank)
    # per-rank workload seeds differ (independent replicas)
    seed = bench.WORKLOAD["seed"] + r
    ms = torch.tensor([10.0 * (rank + 1)])
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    steps = 100
    value = w * steps / (ms.item() / 1e3)
    out.put((rank, seed, ms.item(), value))
    dist.destroy_process_group()


def test_two_rank_replica_timing_is_max_over_ranks():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    rows = sorted(q.get(timeout=10) for _ in range(2))
    assert rows[0][1] != rows[1][1]
    assert rows[0][2] == rows[1][2] == 20.0
    assert rows[0][3] == pytest.approx(2 * 100 / 0.020)
