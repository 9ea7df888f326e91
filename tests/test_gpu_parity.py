"""GPU parity: the CUDA path against the oracle and the reference's golden fixtures.

FP64: bit-exact estimates, iteration counts and outcome flags (integer/byte work, so the
bar is equality).  FP32/FP16: decisions and logical error rate against FP64 within the
stated tolerances.
"""
import zlib

import numpy as np
import pytest

from conftest import load_sim_case

pytestmark = pytest.mark.gpu

NOPP_CASES = ["p050_mi50_nopp_s1", "p040_mi1000_nopp_s106", "p055_mi60_nopp_frz_s21"]


def crc(a):
    return zlib.crc32(np.ascontiguousarray(a, np.uint8).tobytes()) & 0xFFFFFFFF


def opts(**kw):
    from joint_bp_plus_pp_b200 import Options
    base = dict(precision="fp64", enable_pp=False)
    base.update(kw)
    return Options(**base)


def meta_opts(meta, **kw):
    return opts(max_iter=meta["max_iter"], freeze_syn=meta.get("freeze_syn", False), **kw)


@pytest.mark.parametrize("name", NOPP_CASES)
def test_fp64_decode_errors_bit_exact_vs_golden(decoder, name):
    meta, errs, ests = load_sim_case(name)
    st, res, est = decoder.decode_errors(errs, meta["p"], meta_opts(meta))
    recs = meta["records"][:len(errs)]
    assert (est == ests).all()
    assert list(res["iterations"]) == [r["iterations"] for r in recs]
    assert list(res["bp_ok"]) == [r["bp_ok"] for r in recs]
    assert list(res["success"]) == [r["success"] for r in recs]
    assert list(res["exact"]) == [r["exact"] for r in recs]
    assert list(res["stab_equiv"]) == [r["stab_equiv"] for r in recs]


@pytest.mark.parametrize("name", NOPP_CASES)
def test_fp64_simulate_device_mt_sampler_matches_golden(decoder, name):
    """Monte Carlo with the reference error stream generated on the device."""
    meta, _, _ = load_sim_case(name)
    recs = meta["records"]
    first = recs[0]["trial_idx"]
    st, res = decoder.simulate(meta["seed"], len(recs), meta["p"], meta_opts(meta), first_trial=first,
                               sampler="mt19937")
    for r, g in zip(res, recs):
        assert (r["iterations"], r["bp_ok"], r["success"], r["exact"], r["stab_equiv"]) == \
               (g["iterations"], g["bp_ok"], g["success"], g["exact"], g["stab_equiv"]), g["trial_idx"]
    assert st["trials"] == len(recs)
    assert st["failures"] == sum(1 - g["success"] for g in recs)
    assert st["total_iters"] == sum(g["iterations"] for g in recs)


def test_fp64_vs_oracle_fresh_trials(decoder, oracle):
    """Fresh trials at a high error rate (many non-converging trials) against the oracle."""
    from joint_bp_plus_pp_b200 import sample_reference_errors
    for seed, p, mi, k in ((9001, 0.065, 35, 48), (31337, 0.03, 25, 64)):
        err = sample_reference_errors(decoder.n, seed, 1, k, p)
        st, res, est = decoder.decode_errors(err, p, opts(max_iter=mi))
        for t in range(k):
            sx, sz = oracle.syndrome(err[t])
            o = oracle.decode(sx, sz, p, mi, enable_pp=False)
            assert (o["est"] == est[t]).all(), (seed, t)
            assert o["iterations"] == res["iterations"][t]
            assert o["syndrome_ok"] == res["syndrome_ok"][t]


def test_fp64_decode_syndromes(decoder, oracle):
    meta, errs, ests = load_sim_case("p050_mi50_nopp_s1")
    sx = np.stack([oracle.syndrome(e)[0] for e in errs[:8]])
    sz = np.stack([oracle.syndrome(e)[1] for e in errs[:8]])
    st, res, est = decoder.decode_syndromes(sx, sz, meta["p"], meta_opts(meta))
    assert (est == ests[:8]).all()
    assert list(res["iterations"]) == [r["iterations"] for r in meta["records"][:8]]
    assert list(res["syndrome_ok"]) == [r["syndrome_ok"] for r in meta["records"][:8]]


def test_fp64_damping_vs_oracle(decoder, oracle):
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p, mi, d = 0.05, 30, 0.3
    err = sample_reference_errors(decoder.n, 5, 1, 16, p)
    st, res, est = decoder.decode_errors(err, p, opts(max_iter=mi, damping=d))
    for t in range(16):
        sx, sz = oracle.syndrome(err[t])
        o = oracle.decode(sx, sz, p, mi, damping=d, enable_pp=False)
        assert (o["est"] == est[t]).all() and o["iterations"] == res["iterations"][t], t


def test_fp64_freeze_damping_vs_oracle(decoder, oracle):
    """freeze-syn together with damping (the full v2c 4-vectors) and explicit priors."""
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p, mi, d = 0.055, 40, 0.25
    err = sample_reference_errors(decoder.n, 9, 1, 24, p)
    st, res, est = decoder.decode_errors(err, p, opts(max_iter=mi, damping=d, freeze_syn=True))
    for t in range(24):
        sx, sz = oracle.syndrome(err[t])
        o = oracle.decode(sx, sz, p, mi, damping=d, freeze_syn=True, enable_pp=False)
        assert (o["est"] == est[t]).all() and o["iterations"] == res["iterations"][t], t


def test_explicit_prior_equals_p(decoder):
    """A prior passed as probabilities decodes exactly like the prior the decoder derives from p."""
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p = 0.05
    q = [1 - p, p / 3, p / 3, p / 3]
    s = ((q[0] + q[1]) + q[2]) + q[3]
    prior = tuple(x / s for x in q)
    err = sample_reference_errors(decoder.n, 3, 1, 64, p)
    _, r1, e1 = decoder.decode_errors(err, p, opts(max_iter=50))
    _, r2, e2 = decoder.decode_errors(err, 0.3, opts(max_iter=50, prior=prior))
    assert (e1 == e2).all() and (r1["iterations"] == r2["iterations"]).all()


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_llr_freeze_runs(decoder, prec):
    """freeze-syn behind the LLR decoders: outcomes close to FP64 freeze-syn on the same errors."""
    meta, errs, _ = load_sim_case("p055_mi60_nopp_frz_s21")
    s64, r64, _ = decoder.decode_errors(errs, meta["p"], meta_opts(meta), want_est=False)
    slo, rlo, _ = decoder.decode_errors(errs, meta["p"], meta_opts(meta, precision=prec), want_est=False)
    assert slo["trials"] == len(errs)
    assert abs(slo["failures"] - s64["failures"]) <= max(3, len(errs) // 5)


def test_check_interval_schedule(decoder):
    """--cuda-check-interval N: convergence is only tested on iterations warmup + kN or max_iter."""
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p = 0.04
    err = sample_reference_errors(decoder.n, 106, 1, 64, p)
    _, base, _ = decoder.decode_errors(err, p, opts(max_iter=60), want_est=False)
    _, res, _ = decoder.decode_errors(err, p, opts(max_iter=60, check_interval=4, check_warmup=2), want_est=False)
    for b, r in zip(base, res):
        if b["syndrome_ok"]:
            it = r["iterations"]
            assert it == 60 or (it > 2 and (it - 2) % 4 == 0)
            assert it >= b["iterations"]


LLR_ENGINES = [("fp32", "slots"), ("fp16", "slots"), ("fp16", "resident")]


@pytest.mark.parametrize("prec,engine", LLR_ENGINES)
def test_llr_precision_agreement(decoder, prec, engine):
    """FP32/FP16 LLR decoders against FP64 on the same reference-sampled errors at p=0.04."""
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p, k = 0.04, 512
    err = sample_reference_errors(decoder.n, 106, 1, k, p)
    _, r64, e64 = decoder.decode_errors(err, p, opts(max_iter=200))
    _, rlo, elo = decoder.decode_errors(err, p, opts(max_iter=200, precision=prec, engine=engine))
    same = (e64 == elo).all(axis=1)
    assert same.mean() >= 0.99, same.mean()
    assert abs(int(r64["success"].sum()) - int(rlo["success"].sum())) <= 3
    assert np.abs(r64["iterations"].astype(int) - rlo["iterations"].astype(int)).mean() < 0.5


@pytest.mark.parametrize("prec,engine", LLR_ENGINES)
def test_llr_precision_ler_not_worse(decoder, prec, engine):
    """Logical error rate of the LLR decoders is not worse than FP64 within the 95% Wilson
    interval, on the same 8192 reference-sampled errors at p=0.05, max-iter 50 (~3% FER)."""
    from joint_bp_plus_pp_b200 import sample_reference_errors, wilson_interval
    p, k, mi = 0.05, 8192, 50
    err = sample_reference_errors(decoder.n, 2024, 1, k, p)
    s64, r64, _ = decoder.decode_errors(err, p, opts(max_iter=mi), want_est=False)
    slo, rlo, _ = decoder.decode_errors(err, p, opts(max_iter=mi, precision=prec, engine=engine), want_est=False)
    lo64, hi64 = wilson_interval(k, s64["failures"])
    assert s64["failures"] > 50
    assert slo["failures"] / k <= hi64, (slo["failures"], s64["failures"])
    # per-trial outcome disagreement stays small
    assert (r64["success"] != rlo["success"]).mean() < 0.02


def test_device_mt_sampler_equals_host_reference_stream(decoder):
    from joint_bp_plus_pp_b200 import sample_reference_errors
    for seed, p in ((106, 0.04), (2 ** 64 - 3, 0.013)):
        dev = decoder.sample_errors(seed, 1, 40, p, sampler="mt19937")
        host = sample_reference_errors(decoder.n, seed, 1, 40, p)
        assert (dev == host).all()


def test_philox_sampler_statistics(decoder):
    """Device Philox errors: weights and X/Z/Y shares of i.i.d. depolarizing noise."""
    p, k, n = 0.04, 4096, decoder.n
    e = decoder.sample_errors(123, 1, k, p, sampler="philox")
    w = (e != 0).sum(axis=1)
    mean, sd = n * p, (n * p * (1 - p)) ** 0.5
    assert abs(w.mean() - mean) < 5 * sd / k ** 0.5
    assert abs(w.std() - sd) < 0.1 * sd
    counts = np.array([(e == s).sum() for s in (1, 2, 3)], float)
    frac = counts / counts.sum()
    assert np.all(np.abs(frac - 1 / 3) < 5 * (1 / 3 * 2 / 3 / counts.sum()) ** 0.5)
    assert (decoder.sample_errors(123, 1, k, p, sampler="philox") == e).all()       # deterministic
    assert not (decoder.sample_errors(124, 1, 4, p, sampler="philox") == e[:4]).all()  # keyed by seed
    assert (decoder.sample_errors(123, 11, 4, p, sampler="philox") == e[10:14]).all()  # keyed by trial index


def test_simulate_counts_and_hist(decoder):
    st, res = decoder.simulate(106, 2000, 0.04, opts(max_iter=1000, precision="fp32"), hist=True)
    assert st["trials"] == 2000
    assert st["total_iters"] == int(res["iterations"].sum())
    assert int(st["hist"].sum()) == 2000
    assert 7.0 < st["total_iters"] / 2000 < 12.0
    assert st["failures"] <= 2


@pytest.mark.parametrize("prec,engine,tol", [("fp32", "slots", 0.01), ("fp16", "slots", 0.3), ("fp16", "resident", 0.3)])
def test_final_llr_deviation_vs_fp64(decoder, prec, engine, tol):
    """Max |LLR| deviation against FP64 (natural units) after 12 iterations on 256 identical
    trials at p=0.04, over the LLRs inside the LLR decoders' range (|LLR_fp64| <= 50; their
    messages saturate at 110 bits = 76 nat by design), and sign agreement."""
    err = decoder.sample_errors(77, 1, 256, 0.04, sampler="philox")
    it = 12
    _, _, l64 = decoder.decode_errors_llr(err, 0.04, opts(max_iter=it, check_warmup=it))
    _, _, llo = decoder.decode_errors_llr(err, 0.04, opts(max_iter=it, check_warmup=it, precision=prec,
                                                          engine=engine))
    assert np.isfinite(llo).all()
    inside = np.abs(l64) <= 50
    assert np.abs(llo - l64)[inside].max() <= tol
    assert ((llo > 0) != (l64 > 0)).mean() <= 1e-4


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_table_engine_agrees_with_fp64(decoder, prec):
    """The table-driven engine (the mixed-size launch's kernel on this one code) on the shipped
    code: plain BP Philox Monte Carlo in one launch, counters consistent with the records,
    outcomes and iteration counts against FP64 on the same trials."""
    from joint_bp_plus_pp_b200 import Options
    T = 4096
    base = dict(max_iter=200, enable_pp=False)
    st, r = decoder.simulate(606, T, 0.05, Options(precision=prec, engine="table", **base), hist=True)
    assert st["trials"] == T and st["kernel_launches"] == 1
    assert st["failures"] == int((r["success"] == 0).sum()) and st["total_iters"] == int(r["iterations"].sum())
    assert int(st["hist"].sum()) == T
    _, r64 = decoder.simulate(606, T, 0.05, Options(precision="fp64", **base))
    assert (r["success"] == r64["success"]).mean() >= 0.995
    assert (r["iterations"] == r64["iterations"]).mean() >= 0.95
    assert abs(int(r["success"].sum()) - int(r64["success"].sum())) <= 8


def test_table_engine_entry_points_agree(decoder, oracle):
    """Philox Monte Carlo and the same errors given from the host decode identically through
    the table engine; the returned estimates reproduce the reported flags (oracle)."""
    from joint_bp_plus_pp_b200 import Options
    o = Options(precision="fp32", engine="table", max_iter=60, enable_pp=False)
    err = decoder.sample_errors(4242, 11, 64, 0.055, sampler="philox")
    _, r1 = decoder.simulate(4242, 64, 0.055, o, first_trial=11)
    _, r2, est = decoder.decode_errors(err, 0.055, o)
    assert (r1 == r2).all()
    assert 0 < int(r2["syndrome_ok"].sum()) < 64
    for t in range(64):
        ok, exact, stab, success = oracle.classify(err[t], est[t])
        assert (r2["syndrome_ok"][t], r2["exact"][t], r2["success"][t]) == (ok, exact, success), t


def test_table_engine_refuses_other_sources(decoder, oracle):
    from joint_bp_plus_pp_b200 import JbpError, Options
    o = Options(precision="fp32", engine="table", max_iter=20, enable_pp=False)
    err = decoder.sample_errors(1, 1, 4, 0.05)
    sx = np.stack([oracle.syndrome(e)[0] for e in err])
    sz = np.stack([oracle.syndrome(e)[1] for e in err])
    for call in (lambda: decoder.decode_syndromes(sx, sz, 0.05, o),
                 lambda: decoder.simulate(1, 4, 0.05, o, sampler="mt19937"),
                 lambda: decoder.simulate(1, 4, 0.05, Options(precision="fp32", engine="table", enable_pp=True))):
        with pytest.raises(JbpError) as e:
            call()
        assert e.value.code == 4, str(e.value)


def test_sfu_measurement_is_plausible():
    """The SFU microbenchmark behind the roofline denominator: each of ex2, lg2, rcp between a
    quarter and twice 16 results/clk/SM at the device's maximum clock."""
    import torch
    from joint_bp_plus_pp_b200 import measure_sfu
    prop = torch.cuda.get_device_properties(0)
    r = measure_sfu(0)
    ceiling = 16 * prop.multi_processor_count * 2.1   # G/s at a clock up to 2.1 GHz
    for k in ("ex2", "lg2", "rcp"):
        assert 0.25 * ceiling < r[k] < 2.0 * ceiling, (k, r[k])


@pytest.mark.parametrize("warmup,interval", [(0, 1), (3, 2), (0, 4)])
def test_single_trial_path_equals_slot_engine(decoder, oracle, warmup, interval):
    """FP64 decodes of one to three syndromes (the drop-in's cuda_bp_decode calls) run each
    trial's whole BP loop in one cooperative launch (kernels_single.cuh); decisions, iteration
    counts and outcomes equal the slot engine's on the same 64 syndromes, for the test schedule
    given (warmup, interval) and for a caller's explicit prior."""
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Options
    p = 0.045
    err = decoder.sample_errors(77, 1, 64, p)
    sx = np.stack([oracle.syndrome(e)[0] for e in err])
    sz = np.stack([oracle.syndrome(e)[1] for e in err])
    base = Options(precision="fp64", max_iter=200, enable_pp=False, check_warmup=warmup, check_interval=interval)
    _, r_ref, e_ref = decoder.decode_syndromes(sx, sz, p, replace(base, engine="slots"))
    for k in (1, 2, 3):
        for i in range(0, 64, k):
            st, r, e = decoder.decode_syndromes(sx[i:i + k], sz[i:i + k], p, base)
            assert st["kernel_launches"] == len(r) and st["slots"] == 1   # the single-trial path ran
            assert (e == e_ref[i:i + k]).all(), (k, i)
            for f in ("iterations", "syndrome_ok", "success"):
                assert (r[f] == r_ref[i:i + k][f]).all(), (f, k, i)
    q = (1 - p, p / 3, p / 3, p / 3)
    s = ((q[0] + q[1]) + q[2]) + q[3]
    pri = replace(base, prior=tuple(x / s for x in q))
    _, r1, e1 = decoder.decode_syndromes(sx[:2], sz[:2], 0.2, pri)
    _, r2, e2 = decoder.decode_syndromes(sx[:2], sz[:2], 0.2, replace(pri, engine="slots"))
    assert (e1 == e2).all() and (r1["iterations"] == r2["iterations"]).all()


@pytest.mark.parametrize("max_iter,warmup,interval", [(1, 0, 1), (2, 0, 4), (5, 1, 2), (5, 0, 3)])
def test_single_trial_path_short_runs(decoder, oracle, max_iter, warmup, interval):
    """The single-trial path at a few iterations, where the last iteration's test (no check
    phase after it) decides most trials: decisions and records equal the slot engine's."""
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Options
    p = 0.04
    err = decoder.sample_errors(91, 1, 24, p)
    sx = np.stack([oracle.syndrome(e)[0] for e in err])
    sz = np.stack([oracle.syndrome(e)[1] for e in err])
    base = Options(precision="fp64", max_iter=max_iter, enable_pp=False, check_warmup=warmup,
                   check_interval=interval)
    _, r_ref, e_ref = decoder.decode_syndromes(sx, sz, p, replace(base, engine="slots"))
    for i in range(24):
        st, r, e = decoder.decode_syndromes(sx[i:i + 1], sz[i:i + 1], p, base)
        assert st["slots"] == 1
        assert (e[0] == e_ref[i]).all(), i
        for f in ("iterations", "syndrome_ok", "success"):
            assert r[f][0] == r_ref[f][i], (f, i)


def test_staged_small_calls_on_other_engines(decoder, oracle):
    """Calls of one to three syndromes stage their inputs through pinned memory; when the run
    does not take the single-trial path (the slot engine by name, FP16 messages on the resident
    engine, damping) the results come back by the ordinary copies and equal those of one
    batched call."""
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Options
    p = 0.05
    err = decoder.sample_errors(55, 1, 9, p)
    sx = np.stack([oracle.syndrome(e)[0] for e in err])
    sz = np.stack([oracle.syndrome(e)[1] for e in err])
    for o in (Options(precision="fp64", engine="slots", max_iter=100, enable_pp=False),
              Options(precision="fp16", max_iter=100, enable_pp=False),
              Options(precision="fp64", max_iter=100, enable_pp=False, damping=0.25)):
        _, r_all, e_all = decoder.decode_syndromes(sx, sz, p, o)
        for k in (1, 3):
            for i in range(0, 9, k):
                st, r, e = decoder.decode_syndromes(sx[i:i + k], sz[i:i + k], p, o)
                assert (e == e_all[i:i + k]).all(), (o, k, i)
                assert (r["iterations"] == r_all[i:i + k]["iterations"]).all(), (o, k, i)


@pytest.mark.parametrize("warmup,interval", [(0, 1), (3, 2)])
def test_single_trial_fp32_equals_slot_engine(decoder, oracle, warmup, interval):
    """FP32 decodes of one to three syndromes take the single-trial path too (the drop-in's
    cuda_bp_decode with JBP_CUDA_PRECISION=fp32): the slot engine's LLR arithmetic in one
    cooperative launch per trial, so decisions, iteration counts and outcomes equal the slot
    engine's FP32 decoder on the same 48 syndromes."""
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Options
    p = 0.05
    err = decoder.sample_errors(78, 1, 48, p)
    sx = np.stack([oracle.syndrome(e)[0] for e in err])
    sz = np.stack([oracle.syndrome(e)[1] for e in err])
    base = Options(precision="fp32", max_iter=200, enable_pp=False, check_warmup=warmup, check_interval=interval)
    _, r_ref, e_ref = decoder.decode_syndromes(sx, sz, p, replace(base, engine="slots"))
    assert 0 < int(r_ref["syndrome_ok"].sum())
    for k in (1, 2, 3):
        for i in range(0, 48, k):
            st, r, e = decoder.decode_syndromes(sx[i:i + k], sz[i:i + k], p, base)
            assert st["kernel_launches"] == len(r) and st["slots"] == 1   # the single-trial path ran
            assert (e == e_ref[i:i + k]).all(), (k, i)
            for f in ("iterations", "syndrome_ok", "success"):
                assert (r[f] == r_ref[i:i + k][f]).all(), (f, k, i)
    # a caller's explicit prior (the drop-in passes one with every call)
    q = (1 - p, p / 3, p / 3, p / 3)
    s = ((q[0] + q[1]) + q[2]) + q[3]
    pri = replace(base, prior=tuple(x / s for x in q))
    st, r1, e1 = decoder.decode_syndromes(sx[:2], sz[:2], 0.2, pri)
    _, r2, e2 = decoder.decode_syndromes(sx[:2], sz[:2], 0.2, replace(pri, engine="slots"))
    assert st["slots"] == 1 and (e1 == e2).all() and (r1["iterations"] == r2["iterations"]).all()
