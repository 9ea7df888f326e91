"""GPU tests of the trial-resident engine (one thread block per SM holds a whole trial in
shared memory; FP32 arithmetic, FP16 message storage).

It is an LLR decoder, so it is held to the same bars as the slot engine's LLR paths
(test_gpu_parity.py: >= 99% identical estimates and FER within the FP64 Wilson bound); on top,
its integer work is checked exactly: every reported outcome flag is recomputed by the oracle
from the returned estimate, and the same inputs give the same outputs through every entry
point (device sampler, host errors, host syndromes).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ropts(**kw):
    from joint_bp_plus_pp_b200 import Options
    base = dict(precision="fp16", enable_pp=False, engine="resident")
    base.update(kw)
    return Options(**base)


def test_resident_is_one_launch(decoder):
    st, res = decoder.simulate(106, 1000, 0.04, ropts(max_iter=200))
    assert st["trials"] == 1000 and st["kernel_launches"] == 1
    assert st["total_iters"] == int(res["iterations"].sum())


def test_resident_flags_match_oracle_classification(decoder, oracle):
    """At p=0.06 many trials fail; every flag is recomputed from the estimate on the CPU."""
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p, mi, k = 0.06, 40, 96
    err = sample_reference_errors(decoder.n, 77, 1, k, p)
    st, res, est = decoder.decode_errors(err, p, ropts(max_iter=mi))
    assert 0 < int(res["syndrome_ok"].sum()) < k
    for t in range(k):
        ok, exact, stab, success = oracle.classify(err[t], est[t])
        r = res[t]
        assert (r["syndrome_ok"], r["bp_ok"], r["exact"], r["success"]) == (ok, ok, exact, success), t
        if ok:
            assert r["stab_equiv"] == stab and 1 <= r["iterations"] <= mi
        else:
            assert r["iterations"] == mi
    assert st["failures"] == int((res["success"] == 0).sum())
    assert st["exact"] == int(res["exact"].sum())
    assert st["bp_fail"] == int((res["bp_ok"] == 0).sum())


def test_resident_entry_points_agree(decoder, oracle):
    """Device Philox sampler, host errors and host syndromes decode identically."""
    p, mi, k = 0.05, 60, 64
    err = decoder.sample_errors(4242, 11, k, p, sampler="philox")
    st1, r1 = decoder.simulate(4242, k, p, ropts(max_iter=mi), first_trial=11)
    st2, r2, e2 = decoder.decode_errors(err, p, ropts(max_iter=mi))
    assert (r1 == r2).all()
    sx = np.stack([oracle.syndrome(e)[0] for e in err])
    sz = np.stack([oracle.syndrome(e)[1] for e in err])
    _, r3, e3 = decoder.decode_syndromes(sx, sz, p, ropts(max_iter=mi))
    assert (e3 == e2).all()
    assert (r3["iterations"] == r2["iterations"]).all() and (r3["syndrome_ok"] == r2["syndrome_ok"]).all()


def test_resident_mt_sampler_equals_host_stream(decoder):
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p, mi, k = 0.05, 50, 40
    st1, r1 = decoder.simulate(1, k, p, ropts(max_iter=mi), sampler="mt19937")
    _, r2, _ = decoder.decode_errors(sample_reference_errors(decoder.n, 1, 1, k, p), p, ropts(max_iter=mi))
    assert (r1 == r2).all()


def test_resident_check_interval_schedule(decoder):
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p = 0.04
    err = sample_reference_errors(decoder.n, 106, 1, 64, p)
    _, base, _ = decoder.decode_errors(err, p, ropts(max_iter=60), want_est=False)
    _, res, _ = decoder.decode_errors(err, p, ropts(max_iter=60, check_interval=4, check_warmup=2), want_est=False)
    for b, r in zip(base, res):
        if b["syndrome_ok"]:
            it = r["iterations"]
            assert it == 60 or (it > 2 and (it - 2) % 4 == 0)
            assert it >= b["iterations"]


def test_resident_counts_and_hist(decoder):
    st, res = decoder.simulate(106, 4000, 0.04, ropts(max_iter=1000), hist=True)
    assert st["trials"] == 4000
    assert int(st["hist"].sum()) == 4000
    assert st["total_iters"] == int(res["iterations"].sum()) == st["bp_trial_iterations"]
    assert 7.0 < st["total_iters"] / 4000 < 12.0
    assert st["failures"] <= 2


def test_resident_explicit_prior_equals_p(decoder):
    from joint_bp_plus_pp_b200 import sample_reference_errors
    p = 0.05
    q = [1 - p, p / 3, p / 3, p / 3]
    s = ((q[0] + q[1]) + q[2]) + q[3]
    err = sample_reference_errors(decoder.n, 3, 1, 64, p)
    _, r1, e1 = decoder.decode_errors(err, p, ropts(max_iter=50))
    _, r2, e2 = decoder.decode_errors(err, 0.3, ropts(max_iter=50, prior=tuple(x / s for x in q)))
    assert (e1 == e2).all() and (r1["iterations"] == r2["iterations"]).all()


@pytest.mark.parametrize("p", [0.01, 0.025])
def test_resident_fp32_against_fp64_at_low_p(decoder, p):
    """Config 2's lower error rates (the reference's p matrix 0.01 / 0.025 / 0.04, plain BP,
    max-iter 1000): the FP32 trial-resident decoder against the FP64 bit-exact decoder on the
    same 16,384 trials.  Bars: the same outcome on every trial, the same estimate on >= 99.9%
    and the same iteration count on >= 99% of them (the LLR arithmetic may move a convergence
    by an iteration)."""
    from joint_bp_plus_pp_b200 import Options
    k = 16384
    err = decoder.sample_errors(106, 1, k, p, sampler="philox")
    o32 = Options(precision="fp32", engine="resident", max_iter=1000, enable_pp=False)
    o64 = Options(precision="fp64", max_iter=1000, enable_pp=False)
    s32, r32, e32 = decoder.decode_errors(err, p, o32)
    s64, r64, e64 = decoder.decode_errors(err, p, o64)
    assert s32["kernel_launches"] == 1 and s32["trials"] == s64["trials"] == k
    assert (r32["success"] == r64["success"]).all()
    assert (r32["syndrome_ok"] == r64["syndrome_ok"]).all()
    same_est = int((e32 == e64).all(axis=1).sum())
    assert same_est >= 0.999 * k, same_est
    assert int((r32["iterations"] == r64["iterations"]).sum()) >= 0.99 * k
    # the same trials through the device sampler: the resident decoder's outcomes are the same
    _, rs = decoder.simulate(106, k, p, o32, first_trial=1)
    assert (rs["success"] == r32["success"]).all() and (rs["iterations"] == r32["iterations"]).all()


def test_resident_refuses_what_it_does_not_run(decoder):
    from joint_bp_plus_pp_b200 import JbpError
    for bad in (dict(damping=0.2), dict(freeze_syn=True), dict(precision="fp64")):
        with pytest.raises(JbpError) as e:
            decoder.simulate(1, 4, 0.05, ropts(max_iter=10, **bad))
        assert e.value.code == 4


# ---------------------------------------------------------------- post-processing in the resident kernel

@pytest.mark.parametrize("prec", ["fp16", "fp32"])
def test_resident_pp_stage_trials(decoder, oracle, prec):
    """Errors that make each post-processing stage act (constructed trapping-set errors and
    sampled trials), decoded with the stages inside the resident kernel: its flags agree with
    the oracle's classification of its own estimates, and its estimates and records agree with
    the reference's FP64 records on at least 97% and 94% of the cases (the BP before the stages
    is FP32 / FP16)."""
    from test_gpu_pp import gpu_record, golden_record, load_stage_trials
    total = same_est = same_rec = 0
    for (p, mi, fh), cases in sorted(load_stage_trials(decoder.n).items()):
        errs = np.stack([c[1] for c in cases])
        st, res, est = decoder.decode_errors(errs, p, ropts(max_iter=mi, flip_hist=fh, enable_pp=True, precision=prec))
        for (label, err, est_ref, rec), r, e in zip(cases, res, est):
            ok, exact, stab, success = oracle.classify(err, e)
            assert (r["syndrome_ok"], r["exact"], r["success"]) == (ok, exact, success), (label, mi)
            total += 1
            same_est += bool((e == est_ref).all())
            same_rec += gpu_record(r) == golden_record(rec)
    # measured on a B200: same estimate 178 / 181 (FP16 and FP32), same record 172 / 181 (FP16),
    # 175 / 181 (FP32); the rest are trapping-set cases on which the FP32 / FP16 BP before the
    # stages leaves a different state from the FP64 BP, so a stage sees other decisions
    assert same_est >= 0.97 * total, (same_est, total)
    assert same_rec >= 0.94 * total, (same_rec, total)


@pytest.mark.parametrize("prec", ["fp16", "fp32"])
@pytest.mark.parametrize("name", ["p050_mi200_pp_s305", "p060_mi120_pp_s7"])
def test_resident_pp_ler_close_to_fp64(decoder, name, prec):
    from conftest import load_sim_case
    from test_gpu_pp import opts_for
    meta, errs, _ = load_sim_case(name)
    st64, r64, _ = decoder.decode_errors(errs, meta["p"], opts_for(meta), want_est=False)
    st, r, _ = decoder.decode_errors(errs, meta["p"], ropts(max_iter=meta["max_iter"], flip_hist=meta["flip_hist"],
                                                            enable_pp=True, precision=prec), want_est=False)
    assert st["trials"] == len(errs) and st["kernel_launches"] == 1
    # measured on a B200: 0 / 0 failures of 40 (p = 0.05) and 21 / 21 of 24 (p = 0.06), no outcome
    # disagreement, in both precisions
    assert abs(st["failures"] - st64["failures"]) <= 2
    assert (r["success"] != r64["success"]).sum() <= 2


def test_resident_pp_saves_trials(decoder):
    """At p=0.06 with max-iter 120 many trials stall; the in-kernel stages save some of them
    and the Run Summary counters stay consistent with the per-trial records."""
    st, res = decoder.simulate(7, 600, 0.06, ropts(max_iter=120, enable_pp=True))
    assert st["pp_success"] > 0
    assert st["pp_success"] == int(res["pp_success"].sum())
    assert st["failures"] == int((res["success"] == 0).sum())
    assert st["bp_fail"] == int((res["bp_ok"] == 0).sum())
    assert st["flip_pp_success"] == int((res["pp_flip"] & res["success"]).sum())


@pytest.mark.parametrize("engine,prec", [("resident", "fp16"), ("slots", "fp32"), ("slots", "fp64"), ("table", "fp32")])
def test_invalid_error_values_are_rejected(decoder, engine, prec):
    """Error bytes outside 0..3 are found on the device while the errors are read."""
    from joint_bp_plus_pp_b200 import JbpError, Options
    err = np.zeros((3, decoder.n), np.uint8)
    err[1, 4000] = 7
    with pytest.raises(JbpError) as e:
        decoder.decode_errors(err, 0.05, Options(precision=prec, engine=engine, max_iter=5, enable_pp=False))
    assert e.value.code == 1 and "invalid value" in str(e.value)
    st, res, _ = decoder.decode_errors(err[[0, 2]], 0.05, Options(precision=prec, engine=engine, max_iter=5,
                                                                  enable_pp=False))
    assert st["trials"] == 2 and res["success"].all()


@pytest.mark.parametrize("engine,prec", [("resident", "fp16"), ("slots", "fp64")])
def test_pinned_host_inputs_are_read_in_place(decoder, oracle, engine, prec):
    """Errors and syndromes in pinned, device-addressable host memory are read by the kernels
    in place (no staging copy); the results equal those from pageable buffers."""
    import torch
    from joint_bp_plus_pp_b200 import Options
    o = Options(precision=prec, engine=engine, max_iter=60, enable_pp=False)
    err = decoder.sample_errors(515, 1, 300, 0.05, sampler="philox")
    pinned = torch.empty(err.shape, dtype=torch.uint8, pin_memory=True).numpy()
    pinned[:] = err
    s1, r1, e1 = decoder.decode_errors(err, 0.05, o)
    s2, r2, e2 = decoder.decode_errors(pinned, 0.05, o)
    assert (r1 == r2).all() and (e1 == e2).all()
    sx = np.stack([oracle.syndrome(e)[0] for e in err[:64]])
    sz = np.stack([oracle.syndrome(e)[1] for e in err[:64]])
    psx = torch.empty(sx.shape, dtype=torch.uint8, pin_memory=True).numpy()
    psz = torch.empty(sz.shape, dtype=torch.uint8, pin_memory=True).numpy()
    psx[:] = sx
    psz[:] = sz
    _, q1, f1 = decoder.decode_syndromes(sx, sz, 0.05, o)
    _, q2, f2 = decoder.decode_syndromes(psx, psz, 0.05, o)
    assert (q1 == q2).all() and (f1 == f2).all()
    bad = pinned.copy()
    bad_p = torch.empty(err.shape, dtype=torch.uint8, pin_memory=True).numpy()
    bad_p[:] = err
    bad_p[7, 100] = 9
    from joint_bp_plus_pp_b200 import JbpError
    with pytest.raises(JbpError):
        decoder.decode_errors(bad_p, 0.05, o)


def test_autotune_picks_a_configuration_that_decodes_identically(decoder):
    from joint_bp_plus_pp_b200 import Options
    for prec, want in (("fp16", "resident"), ("fp64", "slots"), ("fp32", "slots")):
        o = Options(precision=prec, max_iter=200, enable_pp=False)
        best, rate = decoder.autotune(0.04, o, probe_trials=2048)
        assert rate > 0 and best.engine == want
        s1, r1 = decoder.simulate(9, 512, 0.04, o)
        s2, r2 = decoder.simulate(9, 512, 0.04, best)
        assert (r1["iterations"] == r2["iterations"]).all() and (r1["success"] == r2["success"]).all()


@pytest.mark.parametrize("pp,learned", [(False, 0), (True, 0), (True, 6)])
def test_resident_fp32_messages(decoder, oracle, pp, learned):
    """FP32 messages on the resident tier (asked for explicitly; the messages live in a per-block
    L2-resident scratch): one launch, flags recomputed by the oracle from the returned
    estimates, outcomes against FP64 on the same trials, and AUTO keeps FP32 on the slot engine."""
    from joint_bp_plus_pp_b200 import Options, load_flip_model, sample_reference_errors
    p, k = 0.055, 400
    err = sample_reference_errors(decoder.n, 31, 1, k, p)
    o = Options(precision="fp32", engine="resident", max_iter=200, enable_pp=pp, learned_from=learned)
    decoder.set_flip_model(load_flip_model() if learned else None)
    st, res, est = decoder.decode_errors(err, p, o)
    decoder.set_flip_model(None)
    assert st["trials"] == k and st["kernel_launches"] == 1
    for t in range(0, k, 5):
        ok, exact, stab, success = oracle.classify(err[t], est[t])
        assert (res["syndrome_ok"][t], res["exact"][t], res["success"][t]) == (ok, exact, success), t
    _, r64, _ = decoder.decode_errors(err, p, Options(precision="fp64", max_iter=200, enable_pp=pp), want_est=False)
    assert (res["success"] == r64["success"]).mean() >= 0.98
    assert abs(int(res["success"].sum()) - int(r64["success"].sum())) <= 4
    s_auto, _, _ = decoder.decode_errors(err[:8], p, Options(precision="fp32", max_iter=200, enable_pp=pp))
    assert s_auto["kernel_launches"] > 1          # the slot engine: several launches per run


def test_autotune_can_choose_the_check_interval(decoder):
    """With check_interval 0 (post-processing off) the autotuner also picks the syndrome-test
    interval; the chosen options decode, and trials stop at a multiple of it."""
    from joint_bp_plus_pp_b200 import Options
    o = Options(precision="fp32", max_iter=200, enable_pp=False, check_interval=0)
    best, rate = decoder.autotune(0.04, o, probe_trials=2048)
    assert rate > 0 and best.check_interval in (1, 2, 4)
    st, r = decoder.simulate(9, 512, 0.04, best)
    assert st["trials"] == 512
    done = r["syndrome_ok"] == 1
    assert ((r["iterations"][done] - best.check_warmup) % best.check_interval == 0).all()
    pp, _ = decoder.autotune(0.04, Options(precision="fp16", max_iter=200, enable_pp=True, check_interval=0),
                             probe_trials=1024)
    assert pp.check_interval == 1                     # post-processing keeps a test every iteration
