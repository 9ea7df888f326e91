"""Training recipe of the learned flip proposal (the decoder's own stalled states -> GPU training).

The decoder (resident engine, post-processing on) records, at every stall from iteration
`learned_from` on, the features and labels of the qubits next to an unsatisfied check, of the
qubits whose estimate is wrong and of 1 in 32 of the others (jbp_collect_stall_states).  The
MLP is then trained on the GPU by the library's own forward/backward kernels with Adam
(jbp_mlp_train) and saved as FP32 parameters.

    python -m joint_bp_plus_pp_b200.learned --out data/flip_mlp_params.npy
    python -m joint_bp_plus_pp_b200.learned ablation [--trials N] [--p P ...]   (what it adds)

The default recipe decodes 100,000 seeded depolarizing trials at each p in {0.04, 0.045, 0.05,
0.055} on the shipped [[9216,4612]] code (max-iter 100, flip-hist 5) and records the stalls from
iteration 6 on with at most 30 unsatisfied checks per side -- the states the decoder will
propose on.
"""
import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from . import Decoder, Options, mlp_init, FLIP_MODEL_PATH


def collect(dec, ps=(0.04, 0.045, 0.05, 0.055), trials_per_p=100000, max_iter=100, learned_from=6,
            capacity=2_000_000, seed=20240, flip_hist=5, every=32, precision="fp16"):
    """Stalled states of the decoder itself: at each stall (up to 3 per trial), the qubits next
    to an unsatisfied check, the qubits whose estimate is wrong, and 1 in `every` of the others
    (every = 1: all qubits, so that the labels' rates are those the decoder meets)."""
    xs, ys, info = [], [], []
    o = Options(precision=precision, engine="resident", max_iter=max_iter, enable_pp=True, flip_hist=flip_hist,
                learned_from=learned_from, collect_every=every)
    for i, p in enumerate(ps):
        x, y, st = dec.collect_stall_states(seed + i, trials_per_p, p, o, capacity, first_trial=1)
        xs.append(x)
        ys.append(y)
        info.append({"p": p, "trials": st["trials"], "samples": len(x), "failures": st["failures"],
                     "stalls": int(st["learned_attempts"]) if "learned_attempts" in st else None})
    return np.concatenate(xs), np.concatenate(ys), info


def train(dec, x, y, epochs=12, batch=8192, lr=2e-3, pos_weight=4.0, seed=7):
    params = mlp_init(seed)
    params, hist = dec.mlp_train(params, x, y, epochs=epochs, batch=batch, lr=lr, pos_weight=pos_weight, seed=seed)
    return params, hist


def ablation(dec, ps=(0.045, 0.05, 0.055), trials=32768, seed=808, max_iter=1000, learned_from=6,
             precision="fp32", flip_hist=5, cols=0):
    """What the learned proposal adds, on the same trials of the same decoder (FP32 trial-resident
    BP with ETS / flip / OSD post-processing): (a) "none", no proposal; (b) "llr", the proposal's
    trigger, elimination and acceptance with the columns in the decoder's own |LLR| order (least
    reliable first); (c) "model", the same with the network's order.  Per p and variant:
    trials/s (device time), failures with the Wilson interval, proposals tried and accepted,
    accepted trials that succeed, and mean iterations of the accepted trials; per p, paired LER
    differences of (c) against (b) and (a).  The set model is used for (c); `cols` is the
    proposal's column budget (0 = the default 512)."""
    from . import paired_ler_difference, wilson_interval
    base = dict(precision=precision, engine="resident", max_iter=max_iter, enable_pp=True, flip_hist=flip_hist)
    variants = {"none": Options(**base),
                "llr": Options(learned_from=learned_from, learned_order="llr", learned_cols=cols, **base),
                "model": Options(learned_from=learned_from, learned_cols=cols, **base)}
    out = []
    for p in ps:
        row = {"p": p, "trials": trials, "max_iter": max_iter, "learned_from": learned_from, "cols": cols or 512}
        fails = {}
        for name, o in variants.items():
            dec.simulate(seed, 512, p, o, first_trial=10 ** 9, per_trial=False)   # warm-up
            st, r = dec.simulate(seed, trials, p, o, first_trial=1)
            acc = (r["ets_used_flags"] & 32) != 0
            f = r["success"] == 0
            fails[name] = f
            tried = int(st["learned_attempts"])
            row[name] = {"trials_per_s": trials / (st["device_ms"] / 1e3), "failures": int(f.sum()),
                         "ci95": list(wilson_interval(trials, int(f.sum()))), "attempts": tried,
                         "accepted": int(acc.sum()), "acceptance": int(acc.sum()) / tried if tried else None,
                         "accepted_success": int(st["learned_success"]),
                         "mean_iter_accepted": float(r["iterations"][acc].mean()) if acc.any() else None,
                         "avg_iter": st["total_iters"] / trials}
        for a, b in (("model", "llr"), ("model", "none"), ("llr", "none")):
            d, lo, hi, n10, n01 = paired_ler_difference(fails[a], fails[b])
            row[f"ler_{a}_minus_{b}"] = {"d": d, "ci95": [lo, hi], "fails_only_" + a: n10, "fails_only_" + b: n01}
        out.append(row)
    return out


def main(argv=None):
    if argv is None:
        argv = sys.argv[1:]
    if argv and argv[0] == "ablation":
        ap = argparse.ArgumentParser(prog="python -m joint_bp_plus_pp_b200.learned ablation")
        ap.add_argument("--trials", type=int, default=32768)
        ap.add_argument("--p", type=float, nargs="+", default=[0.045, 0.05, 0.055])
        ap.add_argument("--model", default=str(FLIP_MODEL_PATH))
        ap.add_argument("--cols", type=int, nargs="+", default=[0], help="column budgets (0 = 512)")
        a = ap.parse_args(argv[1:])
        dec = Decoder.from_params()
        dec.set_flip_model(np.load(a.model))
        print(json.dumps([ablation(dec, ps=tuple(a.p), trials=a.trials, cols=c) for c in a.cols], indent=1))
        return 0
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(FLIP_MODEL_PATH))
    ap.add_argument("--trials-per-p", type=int, default=100000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--learned-from", type=int, default=6)
    ap.add_argument("--report", default=None, help="JSON summary of the run")
    ap.add_argument("--p", type=float, nargs="+", default=[0.04, 0.045, 0.05, 0.055])
    ap.add_argument("--collect-every", type=int, default=32,
                    help="record 1 in this many of the quiet, correctly decided qubits (1 = all)")
    ap.add_argument("--capacity", type=int, default=2_000_000, help="samples kept per p at most")
    ap.add_argument("--pos-weight", type=float, default=4.0)
    ap.add_argument("--max-iter", type=int, default=100)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16"],
                    help="message storage of the decoder whose stalls are recorded")
    a = ap.parse_args(argv)
    dec = Decoder.from_params()
    t0 = time.time()
    x, y, info = collect(dec, ps=tuple(a.p), trials_per_p=a.trials_per_p, learned_from=a.learned_from,
                         every=a.collect_every, capacity=a.capacity, max_iter=a.max_iter, precision=a.precision)
    t1 = time.time()
    params, hist = train(dec, x, y, epochs=a.epochs, pos_weight=a.pos_weight)
    t2 = time.time()
    np.save(a.out, params)
    rep = {"samples": int(len(x)), "positives_x": int(y[:, 0].sum()), "positives_z": int(y[:, 1].sum()),
           "collect": info, "collect_s": t1 - t0, "train_s": t2 - t1, "epoch_loss": [float(v) for v in hist],
           "learned_from": a.learned_from, "collect_every": a.collect_every, "pos_weight": a.pos_weight,
           "max_iter": a.max_iter, "precision": a.precision,
           "stalls": int(sum(i["stalls"] or 0 for i in info))}
    print(json.dumps(rep))
    if a.report:
        Path(a.report).write_text(json.dumps(rep, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
