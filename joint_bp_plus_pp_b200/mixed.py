"""Mixed-size Monte Carlo: hypergraph-product codes of seeded random (3,4)-regular classical
codes with classical n in {32, 48, 64, 96} (quantum n 1,600 ... 14,400, variable degrees 3
and 4), depolarizing p drawn per trial uniformly from [p, p_max), decoded together on one
GPU.  Two ways:

* one launch (default): every code's trials in one persistent kernel (jbp_simulate_mixed,
  kernels_mixed.cuh), largest code first;
* concurrent: one context per code, each on its own stream, the calls issued from one host
  thread each so that their kernels run side by side.

    python -m joint_bp_plus_pp_b200.mixed [--trials N] [--precision fp32] [--mode one-launch|concurrent|both]
"""
import argparse
import json
import sys
import threading
import time

from . import Decoder, Options, simulate_mixed as _simulate_mixed
from .codes import hgp_code

CLASSICAL_N = (32, 48, 64, 96)


def build(device=0, classical_n=CLASSICAL_N, seed=7):
    decs = []
    for i, nc in enumerate(classical_n):
        n, xo, xv, zo, zv = hgp_code(nc, seed + i)
        decs.append(Decoder.from_checks(n, xo, xv, zo, zv, device=device))
    return decs


def simulate_one_launch(decs, ntrials, opts, p=0.01, seed=11, first_trial=1, per_trial=False):
    """Every code's Monte Carlo in one kernel launch; returns (per-code stats, wall seconds,
    per-code records or None).  Code i uses seed + i, as simulate_concurrent."""
    k = len(decs)
    t0 = time.perf_counter()
    stats, res = _simulate_mixed(decs, [ntrials] * k, p, opts, seeds=[seed + i for i in range(k)],
                                 first_trial=[first_trial] * k, per_trial=per_trial)
    return stats, time.perf_counter() - t0, res


def simulate_concurrent(decs, ntrials, opts, p=0.01, seed=11, first_trial=1):
    """Runs every code's Monte Carlo at once, one host thread and stream per code; returns
    (per-code stats, wall seconds)."""
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
    ap.add_argument("--mode", default="one-launch", choices=["one-launch", "concurrent", "both"])
    a = ap.parse_args(argv)
    decs = build()
    opts = Options(precision=a.precision, max_iter=a.max_iter, enable_pp=False, p_max=0.06)
    out = {"codes": [d.n for d in decs], "trials_per_code": a.trials}
    modes = ["one-launch", "concurrent"] if a.mode == "both" else [a.mode]
    for mode in modes:
        if mode == "one-launch":
            simulate_one_launch(decs, max(64, a.trials // 16), opts, seed=1000)   # warm-up
            stats, wall, _ = simulate_one_launch(decs, a.trials, opts)
        else:
            simulate_concurrent(decs, max(64, a.trials // 16), opts, seed=1000)
            stats, wall = simulate_concurrent(decs, a.trials, opts)
        total = sum(s["trials"] for s in stats)
        out[mode] = {"trials_per_s": total / wall, "wall_s": wall,
                     "per_code": [{"n": d.n, "trials": s["trials"], "failures": s["failures"],
                                   "avg_iter": s["total_iters"] / max(1, s["trials"]),
                                   "kernel_launches": s["kernel_launches"], "device_ms": s["device_ms"]}
                                  for d, s in zip(decs, stats)]}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
