"""bench.py's replica plumbing on two processes (gloo, CPU): one process per
rank, the barrier around the timed region, and the max over ranks that the
whole-job value is computed from."""
import multiprocessing as mp
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r, w, _ = bench.rank_info()
    dist = bench.dist_setup(w)
    try:
        bench.dist_barrier(dist)
        out.put((r, bench.dist_max(dist, 1.5 * (r + 1))))
        bench.dist_barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_replicas_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 3.0, 1: 3.0}


def test_single_process_needs_no_group():
    import bench
    assert bench.dist_setup(1) is None
    assert bench.dist_max(None, 2.5) == 2.5
