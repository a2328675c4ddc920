"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): barriers,
the max-over-ranks step time and the weak-scaling aggregate.  Reads are
sharded by rank (each rank maps its own batch, pairs kept whole); there is
no data-path collective."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    r, w, local = bench.dist_env()
    d = bench.Dist(w, "gloo")
    d.barrier()
    ms = 100.0 + 25.0 * r  # per-rank step time
    ms_max = d.max(ms)
    value = bench.aggregate_reads_per_s(2_000, w, ms_max)
    shard = bench.shard_seed(r)
    d.barrier()
    d.close()
    q.put((r, local, ms_max, value, shard))


def test_two_rank_max_and_weak_scaling():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    assert all(r[2] == pytest.approx(125.0) for r in res)  # slowest rank's time
    assert all(r[3] == pytest.approx(2 * 2_000 / 0.125) for r in res)  # all ranks' reads / max time
    assert res[0][4] != res[1][4]  # every rank maps different reads
