"""GPU decoding of codes given as check lists with mixed variable degrees (hypergraph products
of random (3,4)-regular classical codes), per-trial error rates, and the mixed-size batch."""
import numpy as np
import pytest

from joint_bp_plus_pp_b200.codes import hgp_code

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hgp():
    from joint_bp_plus_pp_b200 import Decoder
    from oracle_bind import Oracle
    n, xo, xv, zo, zv = hgp_code(32, 1)
    return Decoder.from_checks(n, xo, xv, zo, zv), Oracle.from_checks(n, xo, xv, zo, zv)


@pytest.mark.parametrize("pp", [False, True])
def test_fp64_hgp_bit_exact_vs_oracle(hgp, pp):
    """FP64 on an irregular code (degree-3 and degree-4 variables padded to 4): estimates,
    iteration counts and outcomes equal the oracle's, with and without post-processing."""
    from joint_bp_plus_pp_b200 import Options
    dec, orc = hgp
    p, mi, k = 0.06, 40, 48
    rng = np.random.default_rng(9)
    u = rng.random((k, dec.n))
    err = np.where(u < 1 - p, 0, 1 + ((u - (1 - p)) / p * 3).astype(int).clip(0, 2)).astype(np.uint8)
    st, res, est = dec.decode_errors(err, p, Options(precision="fp64", max_iter=mi, enable_pp=pp))
    assert 0 < int(res["syndrome_ok"].sum()) < k
    for t in range(k):
        o = orc.error_trial(err[t], p, mi, enable_pp=pp)
        assert (o["est"] == est[t]).all(), t
        assert (o["iterations"], o["syndrome_ok"], o["success"]) == \
               (res["iterations"][t], res["syndrome_ok"][t], res["success"][t]), t


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_llr_hgp_agrees_with_fp64(hgp, prec):
    from joint_bp_plus_pp_b200 import Options
    dec, _ = hgp
    err = dec.sample_errors(3, 1, 2000, 0.03, sampler="philox")
    _, r64, e64 = dec.decode_errors(err, 0.03, Options(precision="fp64", max_iter=100, enable_pp=False))
    _, rlo, elo = dec.decode_errors(err, 0.03, Options(precision=prec, max_iter=100, enable_pp=False))
    assert (e64 == elo).all(axis=1).mean() >= 0.98
    assert abs(int(r64["success"].sum()) - int(rlo["success"].sum())) <= 10


def test_per_trial_error_rate_range(hgp):
    """p drawn per trial from [0.01, 0.06): the failure rate lies between those of fixed 0.01
    and 0.06, and the draw is a function of (seed, trial)."""
    from joint_bp_plus_pp_b200 import Options
    dec, _ = hgp
    o = dict(precision="fp32", max_iter=100, enable_pp=False)
    lo, _ = dec.simulate(5, 3000, 0.01, Options(**o), per_trial=False)
    hi, _ = dec.simulate(5, 3000, 0.06, Options(**o), per_trial=False)
    mix, r1 = dec.simulate(5, 3000, 0.01, Options(p_max=0.06, **o))
    _, r2 = dec.simulate(5, 3000, 0.01, Options(p_max=0.06, slots=512, **o))
    assert lo["failures"] <= mix["failures"] <= hi["failures"] and lo["failures"] < hi["failures"]
    assert (r1 == r2).all()


def test_mixed_size_batch_concurrently():
    """The four hypergraph-product codes (n = 1,600 ... 14,400) decoded at once from four host
    threads, each context on its own stream."""
    from joint_bp_plus_pp_b200 import Options
    from joint_bp_plus_pp_b200.mixed import build, simulate_concurrent
    decs = build()
    assert [d.n for d in decs] == [1600, 3600, 6400, 14400]
    opts = Options(precision="fp32", max_iter=200, enable_pp=False, p_max=0.06)
    stats, wall = simulate_concurrent(decs, 1000, opts)
    assert all(s["trials"] == 1000 for s in stats) and wall > 0
    solo, _ = decs[0].simulate(11, 1000, 0.01, opts, per_trial=False)
    assert (solo["failures"], solo["total_iters"]) == (stats[0]["failures"], stats[0]["total_iters"])


@pytest.fixture(scope="module")
def mixed_codes():
    from joint_bp_plus_pp_b200.mixed import build
    return build()


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_mixed_one_launch_agrees_with_fp64(mixed_codes, prec):
    """The four codes (n = 1,600 ... 14,400; the largest keeps its messages in global memory,
    the others in shared memory) in one launch: every code's records are consistent with its
    counters, and its outcomes and iteration counts agree with FP64 BP (slot engine) on the
    same Philox trials with the same per-trial p."""
    from joint_bp_plus_pp_b200 import Options, simulate_mixed
    T, seeds = 600, [21, 22, 23, 24]
    base = dict(max_iter=200, enable_pp=False, p_max=0.04)
    stats, res = simulate_mixed(mixed_codes, [T] * 4, 0.01, Options(precision=prec, **base), seeds=seeds,
                                per_trial=True)
    for d, s, r, seed in zip(mixed_codes, stats, res, seeds):
        assert s["trials"] == T and s["kernel_launches"] == 1
        assert s["failures"] == int((r["success"] == 0).sum())
        assert s["total_iters"] == int(r["iterations"].sum())
        assert s["exact"] == int(r["exact"].sum())
        assert (r["success"] <= r["syndrome_ok"]).all() and (r["exact"] <= r["success"]).all()
        _, r64 = d.simulate(seed, T, 0.01, Options(precision="fp64", **base))
        assert abs(int(r["success"].sum()) - int(r64["success"].sum())) <= max(4, T // 50), d.n
        assert (r["success"] == r64["success"]).mean() >= 0.97, d.n
        assert (r["iterations"] == r64["iterations"]).mean() >= 0.85, d.n


def test_mixed_one_launch_is_per_trial_deterministic(mixed_codes):
    """A code's trials decode the same whatever else shares the launch and in whatever order."""
    from joint_bp_plus_pp_b200 import Options, simulate_mixed
    o = Options(precision="fp32", max_iter=200, enable_pp=False, p_max=0.06)
    _, all4 = simulate_mixed(mixed_codes, [300] * 4, 0.01, o, seeds=[5, 6, 7, 8], per_trial=True)
    _, rev = simulate_mixed(mixed_codes[::-1], [300] * 4, 0.01, o, seeds=[8, 7, 6, 5], per_trial=True)
    _, one = simulate_mixed([mixed_codes[2]], [300], 0.01, o, seeds=[7], per_trial=True)
    for i in range(4):
        assert (all4[i] == rev[3 - i]).all()
    assert (all4[2] == one[0]).all()


def test_mixed_one_launch_refuses_what_it_does_not_run(mixed_codes):
    from joint_bp_plus_pp_b200 import Decoder, JbpError, Options, simulate_mixed
    n, xo, xv, zo, zv = hgp_code(32, 3, dv=3, dc=3)      # checks of weight 6 beside weight 7
    other = Decoder.from_checks(n, xo, xv, zo, zv)
    for decs, o in ((mixed_codes[:2], Options(precision="fp64", enable_pp=False)),
                    (mixed_codes[:2], Options(precision="fp32", enable_pp=True)),
                    ([mixed_codes[0], other], Options(precision="fp32", enable_pp=False))):
        with pytest.raises(JbpError) as e:
            simulate_mixed(decs, [8] * len(decs), 0.02, o)
        assert e.value.code == 4, str(e.value)
    st, _ = simulate_mixed([other], [64], 0.02, Options(precision="fp32", enable_pp=False, max_iter=50))
    assert st[0]["trials"] == 64


def test_cli_decodes_a_check_list_code(tmp_path):
    """bin/jointbp_b200 --checks: a hypergraph-product code from a check-list file, per-trial p."""
    import re
    import subprocess
    from pathlib import Path
    from joint_bp_plus_pp_b200.codes import write_checks
    cli = Path(__file__).resolve().parents[1] / "joint_bp_plus_pp_b200" / "bin" / "jointbp_b200"
    f = tmp_path / "hgp32.checks"
    write_checks(f, *hgp_code(32, 1))
    r = subprocess.run([str(cli), "--checks", str(f), "--simulate", "--p", "0.01", "--p-max", "0.06",
                        "--trials", "2000", "--max-iter", "100", "--precision", "fp32", "--sampler", "philox",
                        "--seed", "3", "--report-every", "0"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    s = dict(re.findall(r"(\w+)=(\S+)", [l for l in r.stdout.splitlines() if l.startswith("trials=")][-1]))
    assert s["trials"] == "2000" and 0 < int(s["failures"]) < 2000


def test_cli_mixed_launch_equals_the_api(tmp_path):
    """bin/jointbp_b200 --mixed: two check-list codes in one launch, per-code Run Summaries equal
    to the C ABI's (same seeds seed + i, same trials)."""
    import re
    import subprocess
    from pathlib import Path
    from joint_bp_plus_pp_b200 import Decoder, Options, simulate_mixed
    from joint_bp_plus_pp_b200.codes import write_checks
    cli = Path(__file__).resolve().parents[1] / "joint_bp_plus_pp_b200" / "bin" / "jointbp_b200"
    files, decs = [], []
    for i, nc in enumerate((16, 32)):
        code = hgp_code(nc, i + 1)
        f = tmp_path / f"hgp{nc}.checks"
        write_checks(f, *code)
        files.append(str(f))
        decs.append(Decoder.from_checks(*code))
    r = subprocess.run([str(cli), "--mixed", ",".join(files), "--simulate", "--no-pp", "--p", "0.01", "--p-max", "0.05",
                        "--trials", "3000", "--max-iter", "100", "--precision", "fp32", "--seed", "40"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("n=")]
    assert len(lines) == 2 and "kernel_launches=1" in r.stdout
    st, _ = simulate_mixed(decs, [3000, 3000], 0.01, Options(precision="fp32", max_iter=100, enable_pp=False,
                                                             p_max=0.05), seeds=[40, 41])
    for line, s in zip(lines, st):
        d = dict(re.findall(r"(\w+)=(\S+)", line))
        assert (int(d["trials"]), int(d["failures"]), int(d["iters"])) == (s["trials"], s["failures"], s["total_iters"])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n_classical", [32, 96])
def test_single_trial_path_on_hgp_codes(n_classical, precision):
    """FP64 and FP32 calls of one and two syndromes (the single-trial cooperative launch) on hypergraph
    products -- checks of weight 7, variables of degree 3 and 4 padded to 4; at classical n = 96
    the code has 14,400 qubits, more than the launch's threads, so threads take a second
    variable and second check rows -- decode as the slot engine does: estimates, iteration
    counts and outcomes."""
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Decoder, Options
    n, xo, xv, zo, zv = hgp_code(n_classical, 1)
    dec = Decoder.from_checks(n, xo, xv, zo, zv)
    p, k = 0.06, 12
    err = dec.sample_errors(21, 1, k, p)
    syn = []
    for side in (0, 1):
        off, var = dec.checks(side)
        bits = (err >> side) & 1
        syn.append((bits[:, var].reshape(k, -1, int(off[1] - off[0])).sum(axis=2) % 2).astype(np.uint8))
    base = Options(precision=precision, max_iter=60, enable_pp=False)
    _, r_ref, e_ref = dec.decode_syndromes(syn[0], syn[1], p, replace(base, engine="slots"))
    for step in (1, 2):
        for i in range(0, k, step):
            st, r, e = dec.decode_syndromes(syn[0][i:i + step], syn[1][i:i + step], p, base)
            assert st["slots"] == 1   # the single-trial path ran
            assert (e == e_ref[i:i + step]).all(), (step, i)
            for f in ("iterations", "syndrome_ok"):
                assert (r[f] == r_ref[i:i + step][f]).all(), (f, step, i)
    dec.close()
