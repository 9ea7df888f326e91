"""GPU post-processing (ETS / flip / OSD, stall detection) against the reference.

FP64 with post-processing enabled must reproduce the reference's per-trial records
(iterations, outcome, which stage saved the trial, ETS usage flags), its estimates and its
Run Summary counters, on the reference's golden fixtures and on trials chosen because they
exercise each stage.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN, load_sim_case

pytestmark = pytest.mark.gpu

PP_CASES = sorted(p.name[4:-5] for p in GOLDEN.glob("sim_*_pp_*.json"))

FIELDS = ("iterations", "bp_ok", "syndrome_ok", "success", "exact", "stab_equiv", "pp_in_decode", "ets_pp_ok",
          "flip_pp_ok", "osd_pp_ok", "used6", "used12", "ets_applied_post", "pp_success_this", "osd_success")


def gpu_record(r):
    f = int(r["ets_used_flags"])
    return {"iterations": int(r["iterations"]), "bp_ok": int(r["bp_ok"]), "syndrome_ok": int(r["syndrome_ok"]),
            "success": int(r["success"]), "exact": int(r["exact"]), "stab_equiv": int(r["stab_equiv"]),
            "pp_in_decode": int(r["pp_in_decode"]), "ets_pp_ok": int(r["pp_ets"]), "flip_pp_ok": int(r["pp_flip"]),
            "osd_pp_ok": int(r["reserved"]), "used6": (f >> 1) & 1, "used12": (f >> 2) & 1,
            "ets_applied_post": (f >> 3) & 1, "pp_success_this": int(r["pp_success"]),
            "osd_success": int(r["pp_osd"])}


def golden_record(g):
    return {k: int(g[k]) for k in FIELDS}


def opts_for(meta, precision="fp64"):
    from joint_bp_plus_pp_b200 import Options
    return Options(precision=precision, max_iter=meta["max_iter"], flip_hist=meta["flip_hist"],
                   enable_pp=meta["enable_pp"], freeze_syn=meta.get("freeze_syn", False))


@pytest.mark.parametrize("name", PP_CASES)
def test_fp64_pp_simulate_matches_reference_records(decoder, name):
    meta, _, _ = load_sim_case(name)
    recs = meta["records"]
    st, res = decoder.simulate(meta["seed"], len(recs), meta["p"], opts_for(meta), first_trial=recs[0]["trial_idx"],
                               sampler="mt19937")
    for r, g in zip(res, recs):
        assert gpu_record(r) == golden_record(g), g["trial_idx"]
    assert st["failures"] == sum(1 - g["success"] for g in recs)
    assert st["pp_success"] == sum(g["pp_success_this"] for g in recs)


@pytest.mark.parametrize("name", PP_CASES)
def test_fp64_pp_estimates_match_reference(decoder, name):
    meta, errs, ests = load_sim_case(name)
    st, res, est = decoder.decode_errors(errs, meta["p"], opts_for(meta))
    assert (est == ests).all()
    for r, g in zip(res, meta["records"][:len(errs)]):
        assert gpu_record(r) == golden_record(g), g["trial_idx"]


def test_fp64_pp_run_summary_matches_reference_cli(decoder):
    cli = json.loads((GOLDEN / "cli_summaries.json").read_text())["p050_mi200_pp_s305_t40"]["summary"]
    meta, _, _ = load_sim_case("p050_mi200_pp_s305")
    st, _ = decoder.simulate(meta["seed"], 40, meta["p"], opts_for(meta), first_trial=1, sampler="mt19937",
                             per_trial=False)
    for key in ("trials", "failures", "bp_fail", "pp_success", "flip_pp_success", "stab_success", "ets_used",
                "ets6_used", "ets12_used"):
        assert st[key] == int(cli[key]), key
    assert st["ets_saved"] == int(cli["ets_saved"])
    assert st["total_iters"] == int(cli["iters"])


def load_stage_trials(n):
    """Reference records on errors that make each post-processing stage act, grouped by
    (p, max_iter, flip_hist) so one GPU call decodes a group."""
    groups = {}
    for c in json.loads((GOLDEN / "pp_stage_trials.json").read_text()):
        e = np.zeros(n, np.uint8)
        for v, s in c["err"]:
            e[v] = s
        est = np.zeros(n, np.uint8)
        for v, s in c["est"]:
            est[v] = s
        groups.setdefault((c["p"], c["max_iter"], c["flip_hist"]), []).append((c["label"], e, est, c["record"]))
    return groups


def test_fp64_pp_stage_trials_match_reference(decoder):
    """Constructed ETS errors and sampled trials on which ETS, flip, OSD and the post-BP ETS
    act: estimates and records equal the reference's."""
    from joint_bp_plus_pp_b200 import Options
    for (p, mi, fh), cases in sorted(load_stage_trials(decoder.n).items()):
        o = Options(precision="fp64", max_iter=mi, flip_hist=fh, enable_pp=True)
        errs = np.stack([c[1] for c in cases])
        st, res, est = decoder.decode_errors(errs, p, o)
        for (label, _, est_ref, rec), r, e in zip(cases, res, est):
            assert (e == est_ref).all(), (label, mi)
            assert gpu_record(r) == golden_record(rec), (label, mi)


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_llr_precisions_with_pp_run(decoder, prec):
    """Post-processing also runs behind the FP32/FP16 decoders (their |LLR| order the OSD)."""
    meta, errs, _ = load_sim_case("p060_mi120_pp_s7")
    st64, r64, _ = decoder.decode_errors(errs, meta["p"], opts_for(meta), want_est=False)
    st, r, _ = decoder.decode_errors(errs, meta["p"], opts_for(meta, prec), want_est=False)
    assert st["trials"] == len(errs)
    assert abs(st["failures"] - st64["failures"]) <= max(3, len(errs) // 4)


def test_us_oscillation_forms_agree_with_the_rule():
    """The one-pass and warp-parallel forms of the us-signal oscillation trigger give the
    reference rule's answer (jointbp_ets.cpp:2021-2053) on 2,000,000 seeded histories, of which
    a good share fire and a good share do not (ramps, i.e. one turn, included)."""
    from joint_bp_plus_pp_b200 import check_us_oscillation
    n = 2_000_000
    bad, fired = check_us_oscillation(n, seed=5)
    assert bad == 0
    assert 0.1 * n < fired < 0.9 * n, fired
