"""The jointbp_cuda.h drop-in: the unmodified reference CLI (jointbp_ets.cpp built with
-DUSE_CUDA, oracle/_ref/jointbp_ets_dropin) linked against lib/libjointbp_cuda.so.

On a GPU its `--cuda` Run Summary must equal the reference CPU run's (golden
cli_summaries.json): the shim decodes with the FP64 engine, which is bit-exact with the CPU
decoder.  Without a GPU the shim reports the failure and the reference program falls back to
its CPU decoder, as it does for its own CUDA build.
"""
import json
import os
import re
import subprocess

import pytest

from conftest import GOLDEN, ROOT

DROPIN = ROOT / "oracle" / "_ref" / "jointbp_ets_dropin"
PARAMS = ROOT / "joint_bp_plus_pp_b200" / "data" / "H_P768_J3_L12_dmax3_nc0-3_1-2_seed11579811919164041.txt"
KEYS = ("trials", "failures", "bp_fail", "pp_success", "stab_success", "iters", "exact_rate")

needs_dropin = pytest.mark.skipif(not DROPIN.exists(), reason="drop-in reference build not present")


def run_dropin(args, env=None):
    e = dict(os.environ)
    if env:
        e.update(env)
    r = subprocess.run([str(DROPIN), "--params", str(PARAMS)] + args, capture_output=True, text=True,
                       cwd=str(PARAMS.parent), env=e, timeout=600)
    line = [l for l in r.stdout.splitlines() if l.startswith("trials=")]
    summary = dict(re.findall(r"(\w+)=(\[[^\]]*\]|\S+)", line[-1])) if line else None
    return r, summary


def golden(name):
    return json.loads((GOLDEN / "cli_summaries.json").read_text())[name]


@needs_dropin
def test_dropin_without_gpu_reports_and_falls_back():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    g = golden("p050_mi50_nopp_s1_t20")
    r, s = run_dropin(g["args"] + ["--cuda"])
    assert r.returncode == 0
    assert "CUDA init failed" in r.stderr
    for k in KEYS:
        assert s[k] == g["summary"][k], k


@pytest.mark.gpu
@needs_dropin
@pytest.mark.parametrize("name", ["p050_mi50_nopp_s1_t200", "p055_mi60_nopp_frz_s21_t60"])
def test_dropin_cuda_run_summary_equals_reference_cpu(name):
    g = golden(name)
    ntr = g["args"][g["args"].index("--trials") + 1]
    args = [a for a in g["args"]]
    args[args.index("--report-every") + 1] = ntr
    r, s = run_dropin(args + ["--cuda"])
    assert r.returncode == 0, r.stderr
    assert "falling back" not in r.stderr and "failed" not in r.stderr, r.stderr
    assert "cuda_k_ms" in r.stdout            # progress report of CUDA-decoded trials
    for k in KEYS:
        assert s[k] == g["summary"][k], (k, s[k], g["summary"][k])


@pytest.mark.gpu
@needs_dropin
def test_dropin_fp32_precision_from_environment():
    g = golden("p050_mi50_nopp_s1_t200")
    r, s = run_dropin(g["args"] + ["--cuda"], env={"JBP_CUDA_PRECISION": "fp32"})
    assert r.returncode == 0 and "failed" not in r.stderr, r.stderr
    assert s["trials"] == g["summary"]["trials"]
    assert abs(int(s["failures"]) - int(g["summary"]["failures"])) <= 3
