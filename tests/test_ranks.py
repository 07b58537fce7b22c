"""The replicas' host plumbing of bench.py on CPU with world size 2 (gloo): the timed region's
milliseconds are combined as the maximum over ranks and the aggregate counts every rank's
work; a rank that fails before the collective makes the other rank's collective end with an
error within the process group's timeout instead of hanging."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    try:
        bench.init_ranks(world, rank, timeout_s=8)
        if rank == fail_rank:
            raise RuntimeError("rank %d fails before its collective" % rank)
        ms = bench.max_over_ranks(100.0 + 50.0 * rank, world)
        q.put((rank, "ok", ms, bench.aggregate_rate(1000, 5, world, ms)))
    except Exception as e:   # reported, not hung
        q.put((rank, "error", type(e).__name__, str(e)[:200]))


def _run(world, fail_rank=-1, limit=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(world):
            r = q.get(timeout=limit)
            out[r[0]] = r[1:]
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()   # the exact processes this test started
    return out


def test_max_over_ranks_and_aggregate():
    out = _run(2)
    assert out[0][0] == "ok" and out[1][0] == "ok"
    assert out[0][1] == out[1][1] == 150.0   # the slowest rank's time
    assert abs(out[0][2] - 2 * 1000 * 5 / 0.150) < 1e-6


def test_a_failing_rank_ends_the_others_collective_with_an_error():
    out = _run(2, fail_rank=1)
    assert out[1][0] == "error"
    assert out[0][0] == "error"   # timeout or closed connection, reported within the limit
