"""bin/jointbp_b200, the reference command line over the batched GPU decoder.

GPU runs are compared with the unmodified reference CLI's Run Summaries and per-trial records
(golden fixtures), including post-processing, which the reference runs only on its CPU path.
"""
import json
import re
import subprocess
import zlib

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, load_sim_case

CLI = ROOT / "joint_bp_plus_pp_b200" / "bin" / "jointbp_b200"
PARAMS = ROOT / "joint_bp_plus_pp_b200" / "data" / "H_P768_J3_L12_dmax3_nc0-3_1-2_seed11579811919164041.txt"
SUMMARY_KEYS = ("trials", "failures", "bp_fail", "pp_success", "flip_pp_success", "stab_success", "ets_used",
                "ets_saved", "ets6_used", "ets6_saved", "ets12_used", "ets12_saved", "fer", "ci95", "iters",
                "avg_iter", "exact_rate")

pytestmark = pytest.mark.skipif(not CLI.exists(), reason="CLI not built")


def run(args, timeout=900):
    r = subprocess.run([str(CLI), "--params", str(PARAMS)] + args, capture_output=True, text=True, timeout=timeout,
                       cwd=str(PARAMS.parent))
    line = [l for l in r.stdout.splitlines() if l.startswith("trials=")]
    s = dict(re.findall(r"(\w+)=(\[[^\]]*\]|\S+)", line[-1])) if line else None
    return r, s


def crc(a):
    return zlib.crc32(np.ascontiguousarray(a, np.uint8).tobytes()) & 0xFFFFFFFF


def test_help_and_usage_errors():
    r = subprocess.run([str(CLI), "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--simulate" in r.stdout
    r = subprocess.run([str(CLI), "--params", str(PARAMS), "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown argument" in r.stderr
    r = subprocess.run([str(CLI), "--simulate"], capture_output=True, text=True)
    assert r.returncode == 1 and "--params is required" in r.stderr
    r = subprocess.run([str(CLI), "--params", str(PARAMS), "--trials", "5"], capture_output=True, text=True)
    assert r.returncode == 1 and "only valid with --simulate" in r.stderr


def test_engine_and_autotune_flags_parse():
    """--engine takes auto / resident / slots / table, --autotune is a flag; a bad engine name is
    a usage error before any GPU work."""
    r = subprocess.run([str(CLI), "--params", str(PARAMS), "--simulate", "--engine", "bogus"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "--engine must be auto, resident, slots or table" in r.stderr
    r = subprocess.run([str(CLI), "--help"], capture_output=True, text=True)
    assert "--engine auto|resident|slots|table" in r.stdout and "--autotune" in r.stdout


def test_mixed_usage_errors(tmp_path):
    r = subprocess.run([str(CLI), "--mixed", "a,b", "--simulate"], capture_output=True, text=True)
    assert r.returncode == 1 and "--mixed decodes with plain BP: add --no-pp" in r.stderr
    r = subprocess.run([str(CLI), "--mixed", "a,b", "--no-pp"], capture_output=True, text=True)
    assert r.returncode == 1 and "--mixed requires --simulate" in r.stderr
    r = subprocess.run([str(CLI), "--mixed", str(tmp_path / "missing.checks"), "--simulate", "--no-pp"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Failed to read checks" in r.stderr


def test_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r, s = run(["--simulate", "--p", "0.05", "--trials", "4", "--seed", "1"])
    assert r.returncode == 1 and "init failed" in r.stderr and s is None


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["p050_mi50_nopp_s1_t200", "p050_mi200_pp_s305_t40", "p055_mi60_nopp_frz_s21_t60",
                                  "p050_mi50_nopp_s1_t1000"])
def test_run_summary_equals_reference(name):
    g = json.loads((GOLDEN / "cli_summaries.json").read_text())[name]
    r, s = run(g["args"] + ["--batch", "64"])
    assert r.returncode == 0, r.stderr
    for k in SUMMARY_KEYS:
        assert s[k] == g["summary"][k], (k, s[k], g["summary"][k])
    # the reference's start-up graph checks line for the shipped code
    assert "hx_hz_orthogonal=true  hx_hz_odd_pairs=0  girth_x=8  girth_z=8" in r.stdout


@pytest.mark.gpu
def test_min_fails_stops_at_the_reference_trial():
    meta, _, _ = load_sim_case("p050_mi50_nopp_s1")
    recs = meta["records"]
    fails = np.cumsum([1 - r["success"] for r in recs])
    cut = int(np.searchsorted(fails, 2) + 1)
    r, s = run(["--simulate", "--p", "0.05", "--max-iter", "50", "--no-pp", "--seed", "1", "--trials", "100000",
                "--min-fails", "2", "--batch", "1024", "--report-every", "0"])
    assert r.returncode == 0, r.stderr
    assert int(s["trials"]) == cut and int(s["failures"]) == 2
    assert int(s["iters"]) == sum(x["iterations"] for x in recs[:cut])


@pytest.mark.gpu
def test_err_and_syndrome_modes(tmp_path, oracle):
    meta, errs, ests = load_sim_case("p050_mi50_nopp_s1")
    k = next(i for i, r in enumerate(meta["records"][:len(errs)]) if not r["success"])
    for i in (0, k):
        ef = tmp_path / f"err{i}.txt"
        ef.write_text("\n".join(str(int(v)) for v in errs[i]) + "\n")
        out = tmp_path / f"est{i}.txt"
        r, _ = run(["--err", str(ef), "--p", "0.05", "--max-iter", "50", "--no-pp", "--est", str(out)])
        ok = meta["records"][i]["success"]
        assert r.returncode == (0 if ok else 2), r.stderr
        assert f"decode_success={'true' if ok else 'false'}" in r.stdout
        est = np.array([int(x) for x in out.read_text().split()], np.uint8)
        assert (est == ests[i]).all()
        sx, sz = oracle.syndrome(errs[i])
        (tmp_path / "sx.txt").write_text("\n".join(map(str, sx)) + "\n")
        (tmp_path / "sz.txt").write_text("\n".join(map(str, sz)) + "\n")
        out2 = tmp_path / f"est_s{i}.txt"
        r, _ = run(["--sx", str(tmp_path / "sx.txt"), "--sz", str(tmp_path / "sz.txt"), "--p", "0.05",
                    "--max-iter", "50", "--no-pp", "--est", str(out2)])
        assert r.returncode in (0, 2), r.stderr
        assert out2.read_text() == out.read_text()


@pytest.mark.gpu
def test_trial_index_with_post_processing():
    """Trial 19 of seed 305 is saved by in-loop flip post-processing in the reference."""
    meta, _, _ = load_sim_case("p050_mi200_pp_s305")
    rec = next(r for r in meta["records"] if r["trial_idx"] == 19)
    assert rec["flip_pp_ok"] == 1
    r, s = run(["--simulate", "--p", "0.05", "--max-iter", "200", "--flip-hist", "5", "--seed", "305",
                "--trials", "1", "--trial-index", "19", "--est", "/dev/stdout"])
    assert r.returncode == 0, r.stderr
    assert int(s["pp_success"]) == 1 and int(s["flip_pp_success"]) == 1 and int(s["iters"]) == rec["iterations"]


@pytest.mark.gpu
def test_resident_engine_and_learned_proposal_from_the_cli(tmp_path):
    """--engine resident with post-processing and the shipped learned model (--learned-from)."""
    base = ["--simulate", "--p", "0.045", "--trials", "8000", "--max-iter", "300", "--flip-hist", "5",
            "--precision", "fp16", "--sampler", "philox", "--seed", "606", "--report-every", "0"]
    r0, s0 = run(base + ["--engine", "resident"])
    assert r0.returncode == 0, r0.stderr
    r1, s1 = run(base + ["--engine", "resident", "--learned-from", "6"])
    assert r1.returncode == 0, r1.stderr
    assert s0["trials"] == s1["trials"] == "8000"
    assert int(s1["failures"]) <= int(s0["failures"]) + 2
    bad = tmp_path / "bad.npy"
    bad.write_bytes(b"not numpy")
    r2, _ = run(base + ["--learned-from", "6", "--flip-model", str(bad)])
    assert r2.returncode != 0 and "npy" in r2.stderr
    r3, _ = run(base + ["--engine", "bogus"])
    assert r3.returncode != 0


@pytest.mark.gpu
@pytest.mark.parametrize("engine,precision", [("slots", "fp64"), ("resident", "fp32")])
def test_iter_hist_out_costs_and_progress_tsv(tmp_path, decoder, engine, precision):
    """--iter-hist-out in the reference's format (jointbp_ets.cpp:4623-4643) with measured costs:
    the fractions sum to 1 and equal the library's histogram of the same trials, the iteration
    cost is positive (CUDA-event device time per trial-iteration), the syndrome-test cost is
    positive on the slot engine and 0 on the resident kernel (the test is fused); and
    --progress-tsv holds the latest line only, in the reference's 12 columns
    (jointbp_ets.cpp:5085-5122), consistent with the Run Summary."""
    from joint_bp_plus_pp_b200 import Options
    h, t = tmp_path / "hist.txt", tmp_path / "progress.tsv"
    k = 3000
    r, s = run(["--simulate", "--p", "0.04", "--trials", str(k), "--max-iter", "200", "--seed", "106", "--sampler",
                "philox", "--precision", precision, "--engine", engine, "--no-pp", "--batch", "1000",
                "--iter-hist-out", str(h), "--progress-tsv", str(t)])
    assert r.returncode == 0, r.stderr
    lines = h.read_text().splitlines()
    assert lines[0].startswith("# costs ") and lines[-len([l for l in lines if not l.startswith("#")]) - 1] == "# iter fraction"
    iter_cost, check_cost = (float(x) for x in lines[0].split()[2:4])
    assert iter_cost > 0.0
    assert (check_cost > 0.0) if engine == "slots" else (check_cost == 0.0)
    assert any(l.startswith("# cost_source " + ("slots" if engine == "slots" else "resident")) for l in lines)
    frac = {int(a): float(b) for a, b in (l.split() for l in lines if not l.startswith("#"))}
    assert abs(sum(frac.values()) - 1.0) < 1e-8
    st, _ = decoder.simulate(106, k, 0.04, Options(precision=precision, engine=engine, max_iter=200, enable_pp=False),
                             per_trial=False, hist=True)
    hist = st["hist"]
    assert set(frac) == {i for i in range(1, len(hist)) if hist[i]}
    for i, f in frac.items():
        assert abs(f - hist[i] / k) < 1e-9, i
    assert abs(sum(i * f for i, f in frac.items()) * k - int(s["iters"])) < 1e-3
    rows = t.read_text().splitlines()
    assert len(rows) == 1   # rewritten after each of the three batches
    cols = rows[0].split("\t")
    assert len(cols) == 12
    assert int(cols[1]) == k and int(cols[2]) == int(s["failures"]) and int(cols[8]) == int(s["iters"])
    assert int(cols[3]) == int(s["pp_success"]) and int(cols[6]) == int(s["stab_success"])
    assert abs(float(cols[7]) - float(s["avg_iter"])) < 0.006
    assert cols[11].startswith(f"PROGRESS | trials={k} | failures={s['failures']} |")


@pytest.mark.gpu
def test_cuda_devices_run_summary_equals_one_device(tmp_path):
    """--cuda-devices splits the trial range over one context and host thread per listed
    device (here device 0 twice: two contexts decoding concurrently on one GPU) and prints one
    merged Run Summary: every key equals the single-context run's, and so does the histogram."""
    args = ["--simulate", "--p", "0.05", "--trials", "20000", "--max-iter", "300", "--seed", "17", "--sampler",
            "philox", "--precision", "fp32", "--engine", "resident", "--flip-hist", "5", "--batch", "4096"]
    r1, s1 = run(args + ["--iter-hist-out", str(tmp_path / "h1.txt")])
    r2, s2 = run(args + ["--cuda-devices", "0,0", "--iter-hist-out", str(tmp_path / "h2.txt")])
    assert r1.returncode == 0 and r2.returncode == 0, r2.stderr
    assert "devices=2" in r2.stdout
    for k in SUMMARY_KEYS:
        assert s1[k] == s2[k], k
    rows = lambda p: [l for l in p.read_text().splitlines() if not l.startswith("#")]
    assert rows(tmp_path / "h1.txt") == rows(tmp_path / "h2.txt")
    assert int(s1["failures"]) > 0
