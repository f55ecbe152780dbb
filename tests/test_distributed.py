"""Multi-process host path of the benchmark (replicas over ranks), on CPU with
gloo and world size 2: each rank gets distinct fields, and the job time is
the slowest rank's device time (MAX over ranks)."""

from __future__ import annotations

import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank
        got = bench.reduce_max_ms(ms, dist, "cpu")
        c = bench.coefficients(16, 2, seed=bench.replica_seed(rank))
        gathered = [None] * world
        dist.all_gather_object(gathered, c[0, :4].tolist())
        q.put((rank, got, gathered))
    finally:
        dist.destroy_process_group()


def test_replicas_max_over_ranks_and_distinct_fields():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, gathered in out:
        assert got == pytest.approx(15.0)  # slowest rank
        assert gathered[0] != gathered[1]  # distinct replica inputs
