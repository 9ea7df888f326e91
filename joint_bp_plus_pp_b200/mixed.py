"""Mixed-size Monte Carlo: hypergraph-product codes of seeded random (3,4)-regular classical
codes with classical n in {32, 48, 64, 96} (quantum n 1,600 ... 14,400, variable degrees 3
and 4), depolarizing p drawn per trial uniformly from [p, p_max), decoded together on one
GPU: one context per code, each on its own stream, the calls issued from one host thread
each so that their kernels run concurrently.

    python -m joint_bp_plus_pp_b200.mixed [--trials N] [--precision fp32]
"""
import argparse
import json
import sys
import threading
import time

from . import Decoder, Options
from .codes import hgp_code

CLASSICAL_N = (32, 48, 64, 96)


def build(device=0, classical_n=CLASSICAL_N, seed=7):
    decs = []
    for i, nc in enumerate(classical_n):
        n, xo, xv, zo, zv = hgp_code(nc, seed + i)
        decs.append(Decoder.from_checks(n, xo, xv, zo, zv, device=device))
    return decs


def simulate_mixed(decs, ntrials, opts, p=0.01, seed=11, first_trial=1):
    """Runs every code's Monte Carlo at once; returns (per-code stats, wall seconds)."""
    out = [None] * len(decs)
    errs = [None] * len(decs)

    def work(i):
        try:
            out[i], _ = decs[i].simulate(seed + i, ntrials, p, opts, first_trial=first_trial, per_trial=False)
        except Exception as e:  # reported below
            errs[i] = e

    ths = [threading.Thread(target=work, args=(i,)) for i in range(len(decs))]
    t0 = time.perf_counter()
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    wall = time.perf_counter() - t0
    for e in errs:
        if e is not None:
            raise e
    return out, wall


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--trials", type=int, default=20000, help="trials per code")
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "fp16"])
    ap.add_argument("--max-iter", type=int, default=200)
    a = ap.parse_args(argv)
    decs = build()
    opts = Options(precision=a.precision, max_iter=a.max_iter, enable_pp=False, p_max=0.06)
    simulate_mixed(decs, max(64, a.trials // 16), opts, seed=1000)   # warm-up
    stats, wall = simulate_mixed(decs, a.trials, opts)
    total = sum(s["trials"] for s in stats)
    print(json.dumps({"codes": [{"n": d.n, "trials": s["trials"], "failures": s["failures"],
                                 "avg_iter": s["total_iters"] / max(1, s["trials"]),
                                 "device_ms": s["device_ms"]} for d, s in zip(decs, stats)],
                      "trials_per_s": total / wall, "wall_s": wall}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
