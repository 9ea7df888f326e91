"""Pins the CPU oracle (oracle/jbp_oracle.c) to the reference.

Golden fixtures under tests/golden/ were produced by the unmodified reference decoder
(tests/golden/make_golden.py); where the reference harness is built (oracle/_ref) the
oracle is also compared with it directly on fresh trials.
"""
import hashlib
import json
import zlib

import numpy as np
import pytest

from conftest import GOLDEN, SIM_CASE_NAMES, load_sim_case
from oracle_bind import Reference, reference_available


def crc(a):
    return zlib.crc32(np.ascontiguousarray(a, np.uint8).tobytes()) & 0xFFFFFFFF


def test_code_known_answers(oracle):
    kat = json.loads((GOLDEN / "kat.json").read_text())
    assert oracle.n == kat["n"] == 9216
    assert oracle.m == (kat["mx"], kat["mz"]) == (2304, 2304)
    xo, xv = oracle.checks(0)
    zo, zv = oracle.checks(1)
    assert hashlib.sha256(xv.astype(np.int32).tobytes()).hexdigest() == kat["x_checks_sha256"]
    assert hashlib.sha256(zv.astype(np.int32).tobytes()).hexdigest() == kat["z_checks_sha256"]
    assert oracle.bx.rank == kat["rank_x"] == 2302
    assert oracle.bz.rank == kat["rank_z"] == 2302
    assert kat["k"] == 4612
    # every X check is orthogonal to every Z check (even overlap), README "hx_hz_orthogonal=true"
    n = oracle.n
    hx = np.zeros((2304, n), np.uint8)
    hz = np.zeros((2304, n), np.uint8)
    for c in range(2304):
        hx[c, xv[xo[c]:xo[c + 1]]] = 1
        hz[c, zv[zo[c]:zo[c + 1]]] = 1
    assert not ((hx.astype(np.int32) @ hz.T.astype(np.int32)) % 2).any()


def test_ets_counts(oracle):
    kat = json.loads((GOLDEN / "kat.json").read_text())
    got = [(lab, cx, cz) for lab, _, cx, cz in oracle.ets_groups()]
    assert got == [(g["label"], g["x"], g["z"]) for g in kat["ets_groups"]]


def test_sampler_golden(oracle):
    kat = json.loads((GOLDEN / "kat.json").read_text())
    for key, exp in kat["sampler"].items():
        seed, p, idx = key.split(":")
        e = oracle.sample(int(seed), int(idx), float(p))
        assert crc(e) == exp["crc"], key
        assert [int((e == s).sum()) for s in range(4)] == exp["counts"]


@pytest.mark.parametrize("name", SIM_CASE_NAMES)
def test_simulate_records_golden(oracle, name):
    meta, errs, ests = load_sim_case(name)
    for k, rec in enumerate(meta["records"]):
        d = oracle.simulate_trial(meta["seed"], rec["trial_idx"], meta["p"], meta["max_iter"],
                                  flip_hist=meta["flip_hist"], enable_pp=meta["enable_pp"],
                                  freeze_syn=meta.get("freeze_syn", False), want_vectors=True)
        err, est = d.pop("err"), d.pop("est")
        exp = dict(rec)
        assert crc(err) == exp.pop("err_crc"), (name, rec["trial_idx"])
        assert crc(est) == exp.pop("est_crc"), (name, rec["trial_idx"])
        assert d == exp, (name, rec["trial_idx"])
        if k < len(errs):
            assert (err == errs[k]).all() and (est == ests[k]).all()


def test_llr_golden(oracle):
    g = np.load(GOLDEN / "llr_golden.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files})
    for key in keys:
        seed, t, mi = key.split("_")
        seed, t, mi = int(seed[1:]), int(t[1:]), int(mi[2:])
        p = 0.05
        err = oracle.sample(seed, t, p)
        sx, sz = oracle.syndrome(err)
        out = oracle.decode(sx, sz, p, mi, enable_pp=False, want_llr=True)
        assert out["iterations"] == int(g[key + "_iters"][0])
        assert (out["est"] == g[key + "_est"]).all()
        assert np.array_equal(out["abs_llr_x"], g[key + "_x"]) and np.array_equal(out["abs_llr_z"], g[key + "_z"])


def test_wilson_matches_cli(oracle):
    cli = json.loads((GOLDEN / "cli_summaries.json").read_text())
    for name, c in cli.items():
        s = c["summary"]
        lo, hi = oracle.wilson(int(s["trials"]), int(s["failures"]))
        exp = s["ci95"].strip("[]").split(",")
        assert f"{lo:.8f}" == exp[0] and f"{hi:.8f}" == exp[1], name


def test_cli_summary_counts_match_records():
    """The golden per-trial records add up to the reference CLI's Run Summary."""
    cli = json.loads((GOLDEN / "cli_summaries.json").read_text())
    meta, _, _ = load_sim_case("p050_mi50_nopp_s1")
    s = cli["p050_mi50_nopp_s1_t200"]["summary"]
    recs = meta["records"]
    assert int(s["failures"]) == sum(1 - r["success"] for r in recs)
    assert int(s["iters"]) == sum(r["iterations"] for r in recs)
    assert int(s["bp_fail"]) == sum(1 - r["bp_ok"] for r in recs)
    meta, _, _ = load_sim_case("p050_mi200_pp_s305")
    s = cli["p050_mi200_pp_s305_t40"]["summary"]
    recs = meta["records"]
    assert int(s["pp_success"]) == sum(r["pp_success_this"] for r in recs)
    assert int(s["flip_pp_success"]) == sum(r["success"] and r["flip_pp_ok"] for r in recs)
    assert int(s["iters"]) == sum(r["iterations"] for r in recs)


@pytest.mark.skipif(not reference_available(), reason="reference harness not built here")
def test_oracle_matches_reference_fresh_trials(oracle):
    ref = Reference()
    cases = [(4242, 0.045, 60, False, 0.0, False, range(1, 13)), (77, 0.058, 110, True, 0.0, False, range(1, 5)),
             (9, 0.055, 40, False, 0.25, True, range(1, 9))]
    for seed, p, mi, pp, damp, frz, idxs in cases:
        for t in idxs:
            a = oracle.simulate_trial(seed, t, p, mi, enable_pp=pp, damping=damp, freeze_syn=frz, want_vectors=True)
            b = ref.simulate_trial(seed, t, p, mi, enable_pp=pp, damping=damp, freeze_syn=frz, want_vectors=True)
            assert (a.pop("est") == b.pop("est")).all()
            assert (a.pop("err") == b.pop("err")).all()
            assert a == b, (seed, t)


def test_pp_stage_trials_golden(oracle):
    """Post-processing stages (in-loop ETS, flip, OSD, post-BP ETS) on the reference's
    stage fixtures: constructed ETS errors and sampled trials that post-processing saves."""
    cases = json.loads((GOLDEN / "pp_stage_trials.json").read_text())
    seen = {"ets_pp_ok": 0, "flip_pp_ok": 0, "osd_success": 0, "ets_applied_post": 0, "used6": 0, "used12": 0}
    for c in cases:
        e = np.zeros(oracle.n, np.uint8)
        for v, s in c["err"]:
            e[v] = s
        d = oracle.error_trial(e, c["p"], c["max_iter"], flip_hist=c["flip_hist"], enable_pp=True)
        est = d.pop("est")
        assert sorted([int(v), int(est[v])] for v in np.nonzero(est)[0]) == sorted(c["est"]), c["label"]
        rec = dict(c["record"])
        rec.pop("trial_idx", None)
        d.pop("trial_idx", None)
        assert d == rec, (c["label"], c["max_iter"])
        for k in seen:
            seen[k] += rec[k]
    assert all(v > 0 for k, v in seen.items() if k != "used12"), seen
