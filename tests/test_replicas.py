"""Multi-GPU runs of bench.py are replicas: every rank runs the whole workload on
its own GPU, with no data-path collective; the job's rate is all ranks' work
over the slowest rank's time.  This checks that aggregation (bench.Dist) with
two gloo ranks on CPU, including ranks that report different times."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    d = bench.Dist()
    try:
        d.barrier()
        # rank r did r + 1 units of work in 1 + r seconds
        rate, t_max = d.aggregate(float(rank + 1), 1.0 + rank)
        q.put((rank, rate, t_max, d.max(float(rank)), d.sum(2.0)))
    finally:
        d.close()


def test_two_gloo_ranks_aggregate_as_replicas():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, rate, t_max, mx, sm in got:
        assert t_max == pytest.approx(2.0)          # the slowest rank
        assert rate == pytest.approx((1 + 2) / 2.0)  # all units / slowest time
        assert mx == 1.0 and sm == 4.0
