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


# ---------------------------------------------------------------- the full Run Summary across ranks

PP_P, PP_MAX_ITER, PP_K = 0.06, 30, 3


def _records_counters(recs, max_iter):
    """jbp_stats counters and the iteration histogram of per-trial records (the reference's
    Run Summary accounting, jointbp_ets.cpp:6212-6245, on the oracle's records)."""
    from joint_bp_plus_pp_b200.runsummary import COUNTERS
    c = dict.fromkeys(COUNTERS, 0)
    hist = [0] * (max_iter + 1)
    for r in recs:
        ok = bool(r["success"])
        c["trials"] += 1
        c["failures"] += not ok
        c["bp_fail"] += not r["bp_ok"]
        c["pp_success"] += r["pp_success_this"]
        c["flip_pp_success"] += ok and r["flip_pp_ok"]
        c["osd_pp_success"] += ok and r["osd_success"]
        c["stab_success"] += ok and not r["exact"] and r["stab_equiv"]
        c["ets_used"] += r["used_any"]
        c["ets6_used"] += r["used6"]
        c["ets12_used"] += r["used12"]
        c["ets_saved"] += ok and r["ets_pp_ok"]
        c["exact"] += r["exact"]
        c["total_iters"] += r["iterations"]
        c["bp_trial_iterations"] += r["iterations"]
        hist[r["iterations"]] += 1
    return c, hist


def _rank_records(oracle, rank):
    first = 1 + rank * PP_K
    return [oracle.simulate_trial(23, t, PP_P, PP_MAX_ITER, enable_pp=True) for t in range(first, first + PP_K)]


def _summary_worker(rank, world, port, q):
    import torch.distributed as dist
    from oracle_bind import Oracle
    from joint_bp_plus_pp_b200.runsummary import merge_run_summaries, run_summary
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c, h = _records_counters(_rank_records(Oracle(), rank), PP_MAX_ITER)
        merged = merge_run_summaries(c, h, group=True)
        q.put((rank, {k: v for k, v in merged.items() if k != "hist"}, merged["hist"].tolist(),
               run_summary(merged)))
    finally:
        dist.destroy_process_group()


def test_run_summary_merged_over_two_ranks_equals_one_process():
    """Every Run Summary counter and the iteration histogram, reduced over two gloo ranks with
    one int64 all-reduce (merge_run_summaries), equal those of one process decoding the union
    of the two trial ranges; both ranks hold the same result."""
    import multiprocessing as mp
    from oracle_bind import Oracle
    from joint_bp_plus_pp_b200.runsummary import merge_run_summaries, run_summary
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_summary_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, c0, h0, s0), (_, c1, h1, s1) = out
    assert c0 == c1 and h0 == h1 and s0 == s1
    oracle = Oracle()
    recs = _rank_records(oracle, 0) + _rank_records(oracle, 1)
    c, h = _records_counters(recs, PP_MAX_ITER)
    single = merge_run_summaries(c, h)
    assert {k: v for k, v in single.items() if k != "hist"} == c0
    assert single["hist"].tolist() == h0
    assert run_summary(single) == s0
    assert s0["trials"] == 2 * PP_K and sum(h0) == 2 * PP_K


@pytest.mark.gpu
def test_run_summary_of_two_ranges_equals_one_run(decoder):
    """On the GPU: two disjoint trial ranges decoded by two calls and merged
    (merge_run_summaries, no process group) give every counter and the histogram of one call
    over their union -- FP32 trial-resident BP+PP with the learned proposal at p = 0.05, where
    failures, post-processing saves and learned proposals all occur."""
    from joint_bp_plus_pp_b200 import Options, load_flip_model
    from joint_bp_plus_pp_b200.runsummary import COUNTERS, merge_run_summaries, run_summary
    decoder.set_flip_model(load_flip_model())
    o = Options(precision="fp32", engine="resident", max_iter=400, enable_pp=True, learned_from=6)
    a, _ = decoder.simulate(31, 6000, 0.05, o, first_trial=1, per_trial=False, hist=True)
    b, _ = decoder.simulate(31, 10000, 0.05, o, first_trial=6001, per_trial=False, hist=True)
    u, _ = decoder.simulate(31, 16000, 0.05, o, first_trial=1, per_trial=False, hist=True)
    merged = merge_run_summaries([a, b])
    one = merge_run_summaries(u)
    for k in COUNTERS:
        if k != "kernel_launches":
            assert merged[k] == one[k], k
    assert (merged["hist"] == one["hist"]).all()
    assert run_summary(merged) == run_summary(one)
    assert one["failures"] > 0 and one["pp_success"] > 0
