"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): each rank decodes its own
disjoint trial range (here with the CPU oracle, since the bench's GPU decode is not available
on this host), and the only cross-rank operations -- max of the time, sum of the counters --
give the same totals as one process decoding the union of the ranges."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

P, MAX_ITER, K, BATCH, WARMUP, STEPS = 0.06, 30, 4, 100, 3, 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_counts(oracle, rank):
    import bench
    first = bench.rank_first_trial(rank, BATCH, WARMUP, STEPS)
    fails = iters = 0
    for t in range(first, first + K):
        rec = oracle.simulate_trial(11, t, P, MAX_ITER, enable_pp=False)
        fails += 1 - rec["success"]
        iters += rec["iterations"]
    return first, {"trials": K, "failures": fails, "iters": iters}


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from oracle_bind import Oracle
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        first, counts = _rank_counts(Oracle(), rank)
        ms, tot = bench.reduce_over_ranks(dist, 10.0 + rank, counts, "cpu")
        q.put((rank, first, ms, tot))
    finally:
        dist.destroy_process_group()


def test_two_ranks_disjoint_ranges_and_reduced_totals():
    import multiprocessing as mp
    import bench
    from oracle_bind import Oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, f0, ms0, tot0), (_, f1, ms1, tot1) = out
    # disjoint ranges: rank 1 starts after rank 0's whole range
    assert f1 - f0 == BATCH * (WARMUP + STEPS + 2) and f1 - f0 >= K
    # max time, summed counters, identical on both ranks
    assert ms0 == ms1 == 11.0 and tot0 == tot1
    oracle = Oracle()
    single = {"trials": 0, "failures": 0, "iters": 0}
    for r in range(2):
        _, c = _rank_counts(oracle, r)
        for k in single:
            single[k] += c[k]
    assert tot0 == single
    assert bench.rank_first_trial(0, BATCH, WARMUP, STEPS) == 1
