#!/usr/bin/env python3
"""Benchmark of the batched joint X/Z BP Monte-Carlo decoder on B200.

Workload (the reference's full post-processing configuration): the shipped [[9216,4612]]
(3,12)-regular APM code with its ETS tables, i.i.d. depolarizing noise p=0.04, max-iter 1000
with per-trial early exit, damping 0, --flip-hist 5, post-processing on (ETS, flip and OSD
in the loop after the stall triggers and after BP), FP32 messages.  The same GPU also runs
the plain FP64 BP+PP decoder on the same workload for the FP32/FP64 ratio.  One step decodes
one batch of `--batch` seeded trials; trial indices never repeat across steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank decodes its own trial range (weak scaling; no collective on the
data path) and rank 0 prints one JSON line.  `--impl reference` times the reference's own
CPU decoder (oracle/_ref/jointbp_ets built from the reference sources, one process per
host core) on the same workload.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PARAMS = ROOT / "joint_bp_plus_pp_b200" / "data" / "H_P768_J3_L12_dmax3_nc0-3_1-2_seed11579811919164041.txt"
REF_BIN = ROOT / "oracle" / "_ref" / "jointbp_ets"
REF_CUDA = {"fp64": ROOT / "oracle" / "_ref" / "jointbp_ets_cuda", "fp32": ROOT / "oracle" / "_ref" / "jointbp_ets_cuda_fp32"}
DROPIN_BIN = ROOT / "oracle" / "_ref" / "jointbp_ets_dropin"
N_QUBITS, EDGES = 9216, 2 * 27648
METRIC = "trials/s at p=0.04 (FP32+learned vs plain FP64 BP+PP, same GPU, equal LER)"
UNIT = "trials/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--batch", type=int, default=131072, help="trials per step")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16", "fp64"],
                    help="message storage: fp32 (FP32 arithmetic and messages), fp16 (FP32 arithmetic with FP16 "
                         "message storage), fp64")
    ap.add_argument("--engine", default=None, choices=["auto", "resident", "slots", "table"],
                    help="default: the trial-resident engine for fp32 / fp16, the slot engine for fp64")
    ap.add_argument("--p", type=float, default=0.04)
    ap.add_argument("--max-iter", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=106)
    ap.add_argument("--no-pp", action="store_true", help="plain BP without post-processing")
    ap.add_argument("--flip-hist", type=int, default=5)
    ap.add_argument("--fp64-batch", type=int, default=131072,
                    help="trials of the FP64 comparison step, the same trials as the first timed step (0 = skip)")
    ap.add_argument("--e2e-batch", type=int, default=65536, help="trials per end-to-end step (0 = skip)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample length")
    ap.add_argument("--slots", type=int, default=0)
    ap.add_argument("--mixed-trials", type=int, default=20000,
                    help="trials per code of the mixed-size one-launch run reported beside (0 = skip)")
    ap.add_argument("--learned-from", type=int, default=6,
                    help="stalled trials try the shipped learned flip proposal from this iteration (0 = off)")
    ap.add_argument("--sweep-trials", type=int, default=131072,
                    help="trials per p of the no-PP sweep p in {0.01, 0.025, 0.04}, FP32 resident against FP64 on "
                         "the same trials (0 = skip)")
    ap.add_argument("--ablation-trials", type=int, default=32768,
                    help="trials per p of the learned-proposal ablation at p 0.045/0.05/0.055: no proposal, the "
                         "|LLR|-ordered proposal, the network (0 = skip)")
    ap.add_argument("--ref-gpu-trials", type=int, default=1000,
                    help="trials of each informative run of the reference's own CUDA path and of this repository's "
                         "drop-in through the reference CLI (--cuda --no-pp; 0 = skip)")
    ap.add_argument("--ler-p", type=float, default=0.05, help="error rate of the failure-bearing LER comparison")
    ap.add_argument("--ler-trials", type=int, default=131072,
                    help="trials of the LER comparison: this decoder against FP64 BP+PP on the same trials (0 = skip)")
    a = ap.parse_args()
    if a.engine is None:
        a.engine = "slots" if a.precision == "fp64" else "resident"
    return a


# ----------------------------------------------------------------------------- helpers

def rank_first_trial(rank, batch, warmup, steps):
    """First trial index of a rank's range: ranks decode disjoint contiguous ranges of
    batch * (warmup + steps + 2) trials (warm-up, timed steps, comparison steps)."""
    return 1 + rank * batch * (warmup + steps + 2)


def reduce_over_ranks(dist, ms, counts, device):
    """Max of the device time over ranks and the sum of integer counters (dict), the only
    cross-rank operations of the bench (no collective on the data path)."""
    import torch
    if dist is None:
        return ms, dict(counts)
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    keys = sorted(counts)
    c = torch.tensor([float(counts[k]) for k in keys], device=device, dtype=torch.float64)
    dist.all_reduce(c)
    return float(t.item()), {k: int(round(v)) for k, v in zip(keys, c.tolist())}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.first = 0

    def mark(self):
        """Start of the timed region: later samples only (the sampler is started before the
        warm-up so that nvidia-smi's own start-up does not fall into the timed region)."""
        self.first = len(self.lines)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[self.first:] or self.lines[-2:]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_rate(p, max_iter, seconds, pp=True, flip_hist=5, procs=None, seed0=1000):
    """Reference CPU decoder, one process per host core, for about `seconds` (trials/s summed)."""
    if not REF_BIN.exists():
        return None
    procs = procs or os.cpu_count() or 1
    # probe the per-process rate with a short run, then size the sample to `seconds`
    probe = _run_ref(p, max_iter, 24, seed0 - 1, pp, flip_hist)
    rate1 = probe[0] / max(probe[1], 1e-9) if probe else 30.0
    trials = max(8, int(rate1 * seconds))
    outs = []
    ths = []
    for k in range(procs):
        th = threading.Thread(target=lambda k=k: outs.append(_run_ref(p, max_iter, trials, seed0 + k, pp, flip_hist)))
        th.start()
        ths.append(th)
    for th in ths:
        th.join()
    outs = [o for o in outs if o]
    if not outs:
        return None
    rate = sum(t / e for t, e, _ in outs if e > 0)
    iters = sum(i for _, _, i in outs)
    return {"value": rate, "unit": UNIT, "cores": len(outs), "kind": "reference",
            "sample": f"{len(outs)} processes x {trials} trials of jointbp_ets --simulate --p {p} --max-iter {max_iter} "
                      f"{_pp_flags(pp, flip_hist)} (distinct seeds), {iters} BP iterations in total"}


def _pp_flags(pp, flip_hist):
    return f"--flip-hist {flip_hist}" if pp else "--no-pp"


def _run_ref(p, max_iter, trials, seed, pp, flip_hist):
    cmd = [str(REF_BIN), "--params", str(PARAMS), "--simulate", "--p", str(p), "--trials", str(trials), "--max-iter",
           str(max_iter), "--seed", str(seed), "--report-every", "0"] + _pp_flags(pp, flip_hist).split()
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=str(PARAMS.parent))
    m = re.search(r"trials=(\d+).*?iters=(\d+).*?elapsed_s=([0-9.]+)s", r.stdout)
    if not m:
        return None
    return int(m.group(1)), float(m.group(3)), int(m.group(2))


# ----------------------------------------------------------------------------- reference arm

def run_reference(args, rank, world):
    if rank != 0:
        return 0
    if not REF_BIN.exists():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU binary oracle/_ref/jointbp_ets not built"}))
        return 0
    per_step = max(2.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_reference_rate(args.p, args.max_iter, per_step / 4, not args.no_pp, args.flip_hist)
    vals = []
    walls = []
    last = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        last = cpu_reference_rate(args.p, args.max_iter, per_step, not args.no_pp, args.flip_hist)
        walls.append((time.perf_counter() - t0) * 1e3)
        vals.append(last["value"])
    value = statistics.median(vals)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.median(walls), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (reference mt19937_64 depolarizing noise)", "impl": "reference",
            "step": "one bounded sample on every host core (the rate probe and the sample itself; wall time)",
            "config": {"workload": workload_name(args, "reference CPU decoder (FP64)"), "p": args.p,
                       "max_iter": args.max_iter, "enable_pp": not args.no_pp, "flip_hist": args.flip_hist},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": last["cores"], "kind": "reference",
                             "sample": last["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


SWEEP_P = (0.01, 0.025, 0.04)


def p_sweep_leg(dec, args, first_trial):
    """Config 2 beside the headline: plain BP (--no-pp) at p in {0.01, 0.025, 0.04}, the FP32
    trial-resident decoder against the FP64 bit-exact decoder on the same Philox trials (the
    reference's own p matrix, job_full.sh).  Rates from the engines' CUDA-event device times."""
    from joint_bp_plus_pp_b200 import Options, paired_ler_difference, wilson_interval
    T = args.sweep_trials
    out = []
    for k, p in enumerate(SWEEP_P):
        first = first_trial + k * T
        o32 = Options(precision="fp32", engine="resident", max_iter=args.max_iter, enable_pp=False)
        o64 = Options(precision="fp64", max_iter=args.max_iter, enable_pp=False)
        # short warm-up runs (buffers, graphs) on other trials
        dec.simulate(args.seed, 4096, p, o32, first_trial=3 * 10 ** 9, per_trial=False)
        dec.simulate(args.seed, 4096, p, o64, first_trial=3 * 10 ** 9, per_trial=False)
        s32, r32 = dec.simulate(args.seed, T, p, o32, first_trial=first)
        s64, r64 = dec.simulate(args.seed, T, p, o64, first_trial=first)
        f32, f64 = r32["success"] == 0, r64["success"] == 0
        d, lo, hi, _, _ = paired_ler_difference(f32, f64)
        v32 = s32["trials"] / (s32["device_ms"] / 1e3)
        v64 = s64["trials"] / (s64["device_ms"] / 1e3)
        out.append({"p": p, "trials": T, "fp32_resident_trials_per_s": v32, "fp64_trials_per_s": v64,
                    "ratio": v32 / v64, "failures_fp32": int(f32.sum()), "failures_fp64": int(f64.sum()),
                    "ci95_fp32": list(wilson_interval(T, int(f32.sum()))),
                    "ci95_fp64": list(wilson_interval(T, int(f64.sum()))),
                    "ler_difference": d, "ler_difference_ci95": [lo, hi],
                    "outcome_disagreements": int((f32 != f64).sum()),
                    "iteration_disagreements": int((r32["iterations"] != r64["iterations"]).sum()),
                    "avg_iter_fp32": s32["total_iters"] / max(1, s32["trials"]),
                    "avg_iter_fp64": s64["total_iters"] / max(1, s64["trials"])})
    return out


def ler_check_leg(dec, args, opts, first_trial):
    """A failure-bearing LER comparison: this run's decoder (opts) against plain FP64 BP+PP on
    the same Philox trials at an error rate where failures occur, with the reference's Wilson
    intervals (jointbp_ets.cpp:4388-4399) and a paired interval on the LER difference."""
    from joint_bp_plus_pp_b200 import Options, paired_ler_difference, wilson_interval
    T, p = args.ler_trials, args.ler_p
    o64 = Options(precision="fp64", max_iter=args.max_iter, enable_pp=True, flip_hist=args.flip_hist)
    sa, ra = dec.simulate(args.seed, T, p, opts, first_trial=first_trial)
    sb, rb = dec.simulate(args.seed, T, p, o64, first_trial=first_trial)
    fa, fb = ra["success"] == 0, rb["success"] == 0
    d, lo, hi, n10, n01 = paired_ler_difference(fa, fb)
    return {"p": p, "trials": T, "max_iter": args.max_iter,
            "this": {"trials_per_s": sa["trials"] / (sa["device_ms"] / 1e3), "failures": int(fa.sum()),
                     "ci95": list(wilson_interval(T, int(fa.sum()))),
                     "learned": {"attempts": sa["learned_attempts"], "saved": sa["learned_success"]},
                     "pp_success": sa["pp_success"]},
            "fp64_bp_pp": {"trials_per_s": sb["trials"] / (sb["device_ms"] / 1e3), "failures": int(fb.sum()),
                           "ci95": list(wilson_interval(T, int(fb.sum()))), "pp_success": sb["pp_success"]},
            "ler_difference": d, "ler_difference_ci95": [lo, hi],
            "interval": "paired Wald interval over the discordant trials",
            "fails_only_this": n10, "fails_only_fp64": n01,
            "outcome_disagreements": int((fa != fb).sum())}


def reference_gpu_leg(args):
    """Informative: the reference's own GPU path (cuda_bp_decode, jointbp_cuda.cu:681-1104, one
    trial at a time, built unmodified for sm_100a in FP64 and in its FP32 form) against this
    repository's drop-in for the same boundary (the unmodified reference CLI built with -DUSE_CUDA
    and linked to lib/libjointbp_cuda.so; FP64, and FP32 LLR messages through
    JBP_CUDA_PRECISION=fp32), on the same command: --simulate --p 0.04 --max-iter 1000
    --no-pp --cuda [--cuda-graph], the reference's mt19937_64 trials.  Rates are the CLI's own
    Run Summary (trials / elapsed_s, host sampling included); failures and iterations come from
    the same summary."""
    out = {}
    runs = [("reference_cuda_fp64", REF_CUDA["fp64"], [], None),
            ("reference_cuda_fp64_graph", REF_CUDA["fp64"], ["--cuda-graph"], None),
            ("reference_cuda_fp32", REF_CUDA["fp32"], [], None),
            ("reference_cuda_fp32_graph", REF_CUDA["fp32"], ["--cuda-graph"], None),
            ("dropin_fp64", DROPIN_BIN, [], None),
            ("dropin_fp32", DROPIN_BIN, [], {"JBP_CUDA_PRECISION": "fp32"})]
    for name, binary, extra, env in runs:
        if not binary.exists():
            out[name] = None
            continue
        cmd = [str(binary), "--params", str(PARAMS), "--simulate", "--p", "0.04", "--trials", str(args.ref_gpu_trials),
               "--max-iter", "1000", "--no-pp", "--cuda", "--seed", str(args.seed), "--report-every", "0"] + extra
        r = subprocess.run(cmd, capture_output=True, text=True, cwd=str(PARAMS.parent), timeout=600,
                           env=dict(os.environ, **env) if env else None)
        m = re.search(r"trials=(\d+) failures=(\d+).*?iters=(\d+).*?elapsed_s=([0-9.]+)s", r.stdout)
        if r.returncode != 0 or not m or "falling back" in r.stderr:
            out[name] = {"error": (r.stderr or r.stdout)[-300:]}
            continue
        t, f, it, el = int(m.group(1)), int(m.group(2)), int(m.group(3)), float(m.group(4))
        out[name] = {"trials": t, "failures": f, "iters": it, "elapsed_s": el, "trials_per_s": t / el,
                     "ms_per_trial": 1e3 * el / t}
    return out


def workload_name(args, decoder, learned_from=0):
    pp = f"BP+PP (ETS, flip, OSD), flip-hist {args.flip_hist}" if not args.no_pp else "plain BP (--no-pp)"
    if learned_from:
        pp += f", learned flip proposal at stalls from iteration {learned_from}"
    return f"batched Monte Carlo, [[9216,4612]] APM code, p={args.p}, max-iter {args.max_iter}, {pp}, {decoder}"


# ----------------------------------------------------------------------------- b200 arm

def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        dist = None
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sys.path.insert(0, str(ROOT))
    from joint_bp_plus_pp_b200 import Decoder, Options, sample_reference_errors, wilson_interval

    dec = Decoder.from_params(device=local)
    pp = not args.no_pp
    from joint_bp_plus_pp_b200 import load_flip_model
    resident_tier = args.precision == "fp16" or (args.precision == "fp32" and args.engine == "resident")
    model = load_flip_model() if (pp and args.learned_from > 0 and resident_tier) else None
    learned_from = args.learned_from if model is not None else 0
    if model is not None:
        dec.set_flip_model(model)
    opts = Options(precision=args.precision, max_iter=args.max_iter, enable_pp=pp, flip_hist=args.flip_hist,
                   slots=args.slots, profile=True, engine=args.engine, learned_from=learned_from)
    B = args.batch
    base = rank_first_trial(rank, B, args.warmup, args.steps)   # distinct trial ranges per rank

    def barrier():
        if dist is not None:
            dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    for w in range(args.warmup):
        # the last warm-up step also sizes the per-trial result buffers the first timed step uses
        dec.simulate(args.seed, B, args.p, opts, first_trial=base + w * B, per_trial=(w == args.warmup - 1))
    torch.cuda.synchronize()
    barrier()
    clocks.mark()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    agg = {"trials": 0, "failures": 0, "total_iters": 0, "check_ms": 0.0, "var_ms": 0.0, "kernel_launches": 0,
           "bp_trial_iterations": 0, "profiled_iterations": 0, "device_ms": 0.0, "pp_success": 0,
           "learned_attempts": 0, "learned_success": 0}
    first_res = None
    step_wall, step_kernel, step_stats = [], [], []
    for k in range(args.steps):
        t0 = time.perf_counter()
        st, res = dec.simulate(args.seed, B, args.p, opts, first_trial=base + (args.warmup + k) * B,
                               per_trial=(k == 0), hist=True)
        step_stats.append(st)
        step_wall.append(round((time.perf_counter() - t0) * 1e3, 2))
        step_kernel.append(round(st["device_ms"], 2))
        if k == 0:
            first_res = res
        for key in agg:
            agg[key] += st[key]
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms, tot = reduce_over_ranks(dist, ev0.elapsed_time(ev1), {"trials": agg["trials"], "failures": agg["failures"]},
                                dev)
    total_trials = float(tot["trials"])
    # the whole job's Run Summary: every counter and the iteration histogram of every rank's
    # timed steps, one int64 all-reduce (outside the timed region)
    from joint_bp_plus_pp_b200.runsummary import merge_run_summaries, run_summary
    merged = merge_run_summaries(step_stats, group=(dist is not None) or None)
    value = total_trials / (ms / 1000.0)

    peak, peak_kind = measured_peaks()
    traffic_tab = json.loads((ROOT / "profiles" / "traffic.json").read_text()) if (ROOT / "profiles" / "traffic.json").exists() else {}
    resident = agg["kernel_launches"] == args.steps and agg["check_ms"] == 0.0
    if resident:
        # trial-resident kernel: no message traffic to HBM; bound by the special-function unit
        # (MUFU: ex2 per edge input, rcp + lg2 per edge output, 1 ex2 + 2 lg2 per coupling)
        mufu_per_ti = 3 * EDGES + 6 * N_QUBITS
        mix = {"ex2": EDGES + 2 * N_QUBITS, "rcp": EDGES, "lg2": EDGES + 4 * N_QUBITS}   # per trial-iteration
        kms = agg["device_ms"]
        msg_bytes = 2 if args.precision == "fp16" else 4
        sm_mhz = clk.get("sm_mhz") or 1965.0
        n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
        derived = 16 * n_sm * sm_mhz / 1e3          # Gop/s: 16 MUFU results / clk / SM
        try:
            from joint_bp_plus_pp_b200 import measure_sfu
            sfu = measure_sfu(local)
            # the rate of the kernel's own mix of the three operations
            sfu_peak = mufu_per_ti / sum(mix[k] / sfu[k] for k in mix)
            sfu_kind = ("measured: MUFU microbenchmark (jbp_measure_sfu) ex2 %.0f, lg2 %.0f, rcp %.0f G/s, at the "
                        "kernel's mix ex2:rcp:lg2 = %d:%d:%d" % (sfu["ex2"], sfu["lg2"], sfu["rcp"], mix["ex2"],
                                                                 mix["rcp"], mix["lg2"]))
            if sfu_peak < 0.5 * derived:
                # a measurement far below the hardware rate (a profiler serialising the
                # microbenchmark, a shared GPU) would inflate the fraction: keep the derived rate
                sfu_kind = (f"derived: 16 MUFU results/clk/SM x {n_sm} SMs x median SM clock {sm_mhz:.0f} MHz "
                            f"(the microbenchmark measured {sfu_peak:.0f} G/s, below half of it)")
                sfu_peak = derived
        except Exception as e:   # the derived figure, said so
            sfu, sfu_peak = None, derived
            sfu_kind = f"derived: 16 MUFU results/clk/SM x {n_sm} SMs x median SM clock {sm_mhz:.0f} MHz ({e})"
        achieved = agg["bp_trial_iterations"] * mufu_per_ti / (kms / 1000.0) / 1e9 if kms > 0 else None
        table = args.engine == "table"
        tr = None if table else traffic_tab.get("resident_dram_bytes_per_trial" if args.precision == "fp16"
                                                else "resident_fp32_dram_bytes_per_trial")
        kname = ("k_mixed (table-driven neighbours, one code, " + args.precision.upper() + " c2v)" if table
                 else "k_resident (trial in shared memory, FP16 c2v)" if args.precision == "fp16"
                 else "k_resident (FP32 c2v: X side in shared memory, Z side in a per-block L2-resident scratch)")
        roofline = {"bound": "sfu", "kernel": kname, "achieved": achieved,
                    "peak": sfu_peak, "unit": "Gop/s", "frac": achieved / sfu_peak if achieved else None,
                    "peak_derived_16_per_clk_sm": derived, "sfu_measured": sfu,
                    "traffic": tr * agg["trials"] / args.steps if tr is not None else None,
                    "peak_kind": sfu_kind,
                    "mufu_ops_per_trial_iteration": mufu_per_ti, "trial_iterations": agg["bp_trial_iterations"],
                    "launches": agg["kernel_launches"], "kernel_ms": kms,
                    # the message traffic an HBM-resident design would move: 4 accesses (read v2c,
                    # write c2v, read c2v, write v2c) per edge and trial-iteration at this run's
                    # message size (4 B FP32, 2 B FP16)
                    "hbm_equivalent_gbs": agg["bp_trial_iterations"] * 4 * EDGES * msg_bytes / (kms / 1000.0) / 1e9,
                    "hbm_equivalent_bytes_per_trial_iteration": 4 * EDGES * msg_bytes,
                    "hbm_peak_gbs": peak}
    else:
        # slot engine: dominant kernel, algorithmic bytes = one read + one write of a message per edge
        es = {"fp32": 4, "fp16": 2, "fp64": 16}[args.precision]
        bytes_per_trial_iter = 2 * EDGES * es          # per kernel (check or variable)
        kname, kms = ("check", agg["check_ms"]) if agg["check_ms"] >= agg["var_ms"] else ("variable", agg["var_ms"])
        achieved = agg["bp_trial_iterations"] * bytes_per_trial_iter / (kms / 1000.0) / 1e9 if kms > 0 else None
        launches = agg["profiled_iterations"]
        traffic = traffic_tab.get(f"{args.precision}_{kname}_bytes_per_trial_iteration")
        if traffic is not None and launches:
            traffic = traffic * agg["bp_trial_iterations"] / launches
        roofline = {"bound": "hbm", "kernel": f"{kname} node ({args.precision})", "achieved": achieved,
                    "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                    "traffic": traffic, "peak_kind": peak_kind, "bytes_per_trial_iteration": bytes_per_trial_iter,
                    "trial_iterations": agg["bp_trial_iterations"], "launches": launches,
                    "check_ms": agg["check_ms"], "var_ms": agg["var_ms"]}

    # FP64 comparison: plain FP64 BP(+PP) on the same GPU, on the trials of the first timed step
    fp64 = None
    if args.fp64_batch > 0 and rank == 0:
        o64 = Options(precision="fp64", max_iter=args.max_iter, enable_pp=pp, flip_hist=args.flip_hist)
        dec.simulate(args.seed, max(32, args.fp64_batch // 16), args.p, o64, first_trial=10 ** 9, per_trial=False)
        torch.cuda.synchronize()
        F = min(args.fp64_batch, B)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        st64, r64 = dec.simulate(args.seed, F, args.p, o64, first_trial=base + args.warmup * B)
        b.record()
        torch.cuda.synchronize()
        rlo = first_res[:F]
        f64, flo = int(st64["failures"]), int((rlo["success"] == 0).sum())
        fp64 = {"value": st64["trials"] / (a.elapsed_time(b) / 1000.0), "trials": st64["trials"],
                "failures": f64, "ci95": list(wilson_interval(F, f64)),
                "avg_iter": st64["total_iters"] / max(1, st64["trials"]),
                "same_trials": {"trials": F, "failures_this": flo, "failures_fp64": f64,
                                "ci95_this": list(wilson_interval(F, flo)),
                                "outcome_disagreements": int((rlo["success"] != r64["success"]).sum()),
                                "iteration_disagreements": int((rlo["iterations"] != r64["iterations"]).sum()),
                                "ler_difference": (flo - f64) / F}}

    # precision report: final LLRs against FP64 on identical trials with a fixed iteration count
    precision = None
    if args.fp64_batch > 0 and rank == 0 and args.precision != "fp64":
        it = 12
        perr = dec.sample_errors(args.seed, base + 7 * 10 ** 8, 256, args.p, sampler="philox")
        base_o = dict(max_iter=it, check_warmup=it, enable_pp=False)
        _, r64p, l64 = dec.decode_errors_llr(perr, args.p, Options(precision="fp64", **base_o))
        _, rlop, llo = dec.decode_errors_llr(perr, args.p, Options(precision=args.precision, engine=args.engine,
                                                                   **base_o))
        inside = np.abs(l64) <= 50
        dev = np.abs(llo - l64)
        anyin = bool(inside.any())   # at low p every LLR can have grown past the range in 12 iterations
        precision = {"trials": 256, "iterations": it, "llr_entries": int(l64.size),
                     "llr_entries_compared": int(inside.sum()),
                     "max_abs_llr_dev_nat": float(dev[inside].max()) if anyin else None,
                     "max_rel_llr_dev": float((dev[inside] / np.maximum(np.abs(l64[inside]), 1.0)).max())
                     if anyin else None,
                     "range": "|LLR_fp64| <= 50 nat (messages saturate at 110 bits = 76 nat)",
                     "sign_disagreements": int(((llo > 0) != (l64 > 0)).sum())}

    # config 3 beside the headline: the mixed-size workload in one launch (rank 0)
    mixed = None
    if args.mixed_trials > 0 and rank == 0:
        try:
            from joint_bp_plus_pp_b200.mixed import build as build_mixed, simulate_one_launch
            mdecs = build_mixed(device=local)
            mo = Options(precision="fp32", max_iter=200, enable_pp=False, p_max=0.06)
            simulate_one_launch(mdecs, max(64, args.mixed_trials // 16), mo, seed=1000)   # warm-up
            mst, mwall, _ = simulate_one_launch(mdecs, args.mixed_trials, mo)
            mtot = sum(x["trials"] for x in mst)
            mixed = {"workload": "hypergraph-product codes of seeded random (3,4)-regular classical codes, classical "
                                 "n 32/48/64/96 (n 1,600-14,400), p uniform in [0.01, 0.06) per trial, max-iter 200, "
                                 "plain BP, FP32 messages, all codes in one kernel launch",
                     "trials_per_s": mtot / mwall, "device_trials_per_s": mtot / (mst[0]["device_ms"] / 1000.0),
                     "launches": mst[0]["kernel_launches"],
                     "per_code": [{"n": d.n, "trials": x["trials"], "failures": x["failures"],
                                   "avg_iter": x["total_iters"] / max(1, x["trials"])} for d, x in zip(mdecs, mst)]}
            del mdecs
        except Exception as e:   # reported, the headline line still prints
            mixed = {"error": str(e)}

    # end to end through the C ABI with host buffers (reference-sampled errors in pinned memory)
    e2e = None
    if args.e2e_batch > 0:
        E = args.e2e_batch
        host = torch.empty((E, N_QUBITS), dtype=torch.uint8, pin_memory=True).numpy()
        host[:] = sample_reference_errors(N_QUBITS, args.seed, base + 5 * 10 ** 8, E, args.p)
        oe = Options(precision=args.precision, max_iter=args.max_iter, enable_pp=pp, flip_hist=args.flip_hist,
                     slots=args.slots, engine=args.engine, learned_from=learned_from)
        dec.decode_errors(host[: max(32, E // 8)], args.p, oe, want_est=False)
        torch.cuda.synchronize()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        nsteps = max(1, min(args.steps, 3))
        done = e2e_launches = 0
        for _ in range(nsteps):
            st, res, _ = dec.decode_errors(host, args.p, oe, want_est=False)
            done += st["trials"]
            e2e_launches += st["kernel_launches"]
        b.record()
        torch.cuda.synchronize()
        ems, tot_e = reduce_over_ranks(dist, a.elapsed_time(b), {"trials": done}, dev)
        done = tot_e["trials"]
        e2e = {"value": done / (ems / 1000.0), "unit": UNIT, "h2d_bytes_per_step": E * N_QUBITS,
               "d2h_bytes_per_step": E * 16, "path": "jbp_decode_errors (host errors, pinned) -> results to host",
               "steps": nsteps, "gpu_launches": e2e_launches}

    # config 2's p sweep (no PP) and a failure-bearing LER comparison, both on trials no other
    # leg decodes (rank 0)
    p_sweep = ler_check = None
    if rank == 0 and args.sweep_trials > 0:
        t0 = time.perf_counter()
        p_sweep = {"points": p_sweep_leg(dec, args, 4 * 10 ** 9), "wall_s": None}
        p_sweep["wall_s"] = round(time.perf_counter() - t0, 2)
    if rank == 0 and args.ler_trials > 0:
        t0 = time.perf_counter()
        ler_check = ler_check_leg(dec, args, opts, 5 * 10 ** 9)
        ler_check["wall_s"] = round(time.perf_counter() - t0, 2)
    ref_gpu = None
    if rank == 0 and args.ref_gpu_trials > 0:
        t0 = time.perf_counter()
        ref_gpu = {"runs": reference_gpu_leg(args), "wall_s": None}
        ref_gpu["wall_s"] = round(time.perf_counter() - t0, 2)
    ablation = None
    if rank == 0 and args.ablation_trials > 0 and model is not None and args.precision == "fp32":
        from joint_bp_plus_pp_b200.learned import ablation as learned_ablation
        t0 = time.perf_counter()
        ablation = {"points": learned_ablation(dec, trials=args.ablation_trials, max_iter=args.max_iter,
                                               learned_from=args.learned_from),
                    "wall_s": None}
        ablation["wall_s"] = round(time.perf_counter() - t0, 2)

    cpu = None
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        cpu = cpu_reference_rate(args.p, args.max_iter, args.cpu_seconds, pp, args.flip_hist)

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    lo, hi = wilson_interval(merged["trials"], merged["failures"])
    
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp32": "f32", "fp16": "f32 arithmetic, f16 message storage", "fp64": "f64"}[args.precision],
        "data": "synthetic: Philox4x32-10 depolarizing noise keyed by (seed, trial index)",
        "config": {"workload": workload_name(args, {"fp16": "FP32 arithmetic with FP16 message storage",
                                                    "fp32": "FP32 messages", "fp64": "FP64 messages"}[args.precision],
                                             learned_from),
                   "p": args.p,
                   "max_iter": args.max_iter, "enable_pp": pp, "flip_hist": args.flip_hist,
                   "learned_from": learned_from,
                   "learned": {"attempts": agg["learned_attempts"], "saved": agg["learned_success"]},
                   "trials_per_step": B,
                   "engine": "table" if args.engine == "table" else ("resident" if resident else "slots"),
                   "l2": ("messages in a per-block scratch of 32 MB in all (FP32), L2-resident; variable totals "
                          "in shared memory" if args.engine == "table" and args.precision == "fp32"
                          else "X-side FP32 messages and the rest of the trial in shared memory, Z-side FP32 messages "
                               "in a per-block scratch of 16 MB in all, L2-resident" if resident and args.precision == "fp32"
                          else "trial state in shared memory; no message traffic to HBM" if resident
                          else "message state (>= 7 GB) larger than L2"),
                   "parallelism": f"replica trial ranges x{world}"},
        "gpu_launches": agg["kernel_launches"],
        "roofline": roofline,
        "ler": {"trials": merged["trials"], "failures": merged["failures"], "ci95": [lo, hi],
                "avg_iter": merged["total_iters"] / max(1, merged["trials"])},
        "run_summary": dict(run_summary(merged), ranks=world,
                            iter_hist_nonzero={int(i): int(c) for i, c in enumerate(merged["hist"]) if c}),
        "fp64": fp64,
        "precision": precision,
        "mixed_sizes_one_launch": mixed,
        "p_sweep": p_sweep,
        "ler_check": ler_check,
        "learned_ablation": ablation,
        "informative": {"reference_gpu_path": ref_gpu},
        "clocks": clk,
        "step_ms": {"host_wall": step_wall, "kernel": step_kernel},
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    if fp64:
        line["fp32_over_fp64"] = value / fp64["value"]
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
