"""Run Summary of a Monte Carlo run split over ranks, devices or calls.

Trials are independent and keyed by (seed, trial index), so a run split into disjoint trial
ranges -- one per rank under torch.distributed, one per device, or one per call -- has the
Run Summary of the whole run once its counters are summed.  `merge_run_summaries` does that
with one int64 all-reduce (sum) of every counter of jbp_stats and the iteration histogram
(max_iter + 1 bins) when a process group is given; `run_summary` turns the merged counters
into the reference's Run Summary keys (jointbp_ets.cpp:6414-6449) with its Wilson interval
(jointbp_ets.cpp:4388-4399).
"""
import numpy as np

from . import STAT_FIELDS, wilson_interval

# every integer counter of jbp_stats (include/jbp_b200.h), in one fixed order
COUNTERS = tuple(STAT_FIELDS) + ("bp_trial_iterations", "learned_attempts", "learned_success", "kernel_launches",
                                 "syndrome_tests")


def merge_run_summaries(stats, hist=None, group=None, max_iter=None):
    """Sums the counters (and histograms) of several runs of this process and, with a
    torch.distributed process group `group` (or the default group when `group` is True), of
    every rank.  `stats`: one jbp_stats dict or a list of them; `hist`: None, one histogram or
    a list of them (as returned by Decoder.simulate(hist=True) in stats["hist"] when None).
    Every rank must call this with the same histogram length (max_iter + 1).  Returns a dict of
    the summed counters with "hist" (int64 array) when histograms were given."""
    runs = [stats] if isinstance(stats, dict) else list(stats)
    if hist is None:
        hists = [r["hist"] for r in runs if "hist" in r]
    elif np.ndim(hist) == 1 and len(hist) and np.isscalar(hist[0]):
        hists = [hist]   # one histogram
    else:
        hists = list(hist)
    nbins = max([len(h) for h in hists], default=0)
    if max_iter is not None:
        nbins = max(nbins, max_iter + 1)
    vec = np.zeros(len(COUNTERS) + nbins, np.int64)
    for r in runs:
        vec[:len(COUNTERS)] += np.array([int(r.get(k, 0)) for k in COUNTERS], np.int64)
    for h in hists:
        vec[len(COUNTERS):len(COUNTERS) + len(h)] += np.asarray(h, np.int64)
    if group is not None and group is not False:
        import torch
        import torch.distributed as dist
        g = None if group is True else group
        nccl = dist.get_backend(g) == "nccl"
        t = torch.from_numpy(vec)
        if nccl:
            t = t.to(torch.device("cuda", torch.cuda.current_device()))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=g)
        vec = t.cpu().numpy()
    out = {k: int(v) for k, v in zip(COUNTERS, vec[:len(COUNTERS)])}
    if nbins:
        out["hist"] = vec[len(COUNTERS):].copy()
    return out


def run_summary(merged):
    """The reference Run Summary keys of merged counters: trials, failures, bp_fail,
    pp_success, flip_pp_success, stab_success, the ETS counters, fer, ci95 (Wilson, z = 1.96),
    iters, avg_iter, exact_rate."""
    d = int(merged["trials"])
    out = {k: int(merged[k]) for k in ("trials", "failures", "bp_fail", "pp_success", "flip_pp_success",
                                       "stab_success", "ets_used", "ets_saved", "ets6_used", "ets6_saved",
                                       "ets12_used", "ets12_saved")}
    out["fer"] = merged["failures"] / d if d else 0.0
    out["ci95"] = list(wilson_interval(d, int(merged["failures"]))) if d else None
    out["iters"] = int(merged["total_iters"])
    out["avg_iter"] = merged["total_iters"] / d if d else 0.0
    out["exact_rate"] = merged["exact"] / d if d else 0.0
    return out
