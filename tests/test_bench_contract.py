"""bench.py's host-side contract, on CPU: the reference arm's JSON line (the keys the
reported comparison reads), its behaviour off rank 0 and without the reference binary, the
parse of the reference CLI's run summary, the clock record built from nvidia-smi samples
(the throttle reasons that decide whether a timed run stands), and the Wilson interval of the
reported failure counts."""
import json
import sys
import types
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _args(**kw):
    d = dict(gpus=1, steps=3, warmup=3, p=0.04, max_iter=1000, no_pp=False, flip_hist=5)
    d.update(kw)
    return types.SimpleNamespace(**d)


def test_reference_arm_line(monkeypatch, capsys):
    calls = []

    def fake_rate(p, max_iter, seconds, pp=True, flip_hist=5, procs=None, seed0=1000):
        calls.append((p, max_iter, seconds, pp, flip_hist))
        return {"value": 100.0 + len(calls), "unit": bench.UNIT, "cores": 4, "kind": "reference",
                "sample": "fake sample"}

    monkeypatch.setattr(bench, "cpu_reference_rate", fake_rate)
    monkeypatch.setattr(bench, "REF_BIN", ROOT / "bench.py")     # any file that exists
    assert bench.run_reference(_args(), 0, 1) == 0
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["steps"] == 3 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["higher_is_better"] is True and line["vs_baseline"] is None
    # three warm-up samples, then three timed ones, all of the configured workload
    assert len(calls) == 6
    assert all(c[0] == 0.04 and c[1] == 1000 and c[3] is True and c[4] == 5 for c in calls)
    assert line["value"] == 105.0                                    # median of 104, 105, 106
    assert line["cpu_baseline"] == {"value": 105.0, "unit": bench.UNIT, "cores": 4, "kind": "reference",
                                    "sample": "fake sample"}
    assert line["e2e"] == {"value": 105.0, "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert isinstance(line["ms_per_step"], float) and line["ms_per_step"] >= 0.0
    assert line["config"]["p"] == 0.04 and line["config"]["enable_pp"] is True


def test_reference_arm_no_pp_workload(monkeypatch, capsys):
    seen = []
    monkeypatch.setattr(bench, "cpu_reference_rate",
                        lambda p, mi, s, pp=True, fh=5, **k: seen.append(pp) or
                        {"value": 1.0, "unit": bench.UNIT, "cores": 1, "kind": "reference", "sample": "x"})
    monkeypatch.setattr(bench, "REF_BIN", ROOT / "bench.py")
    assert bench.run_reference(_args(no_pp=True, steps=1, warmup=0), 0, 1) == 0
    line = json.loads(capsys.readouterr().out.strip())
    assert seen == [False] and line["config"]["enable_pp"] is False
    assert "--no-pp" in line["config"]["workload"]


def test_reference_arm_other_ranks_print_nothing(monkeypatch, capsys):
    def boom(*a, **k):
        raise AssertionError("a rank other than 0 ran the reference decoder")

    monkeypatch.setattr(bench, "cpu_reference_rate", boom)
    assert bench.run_reference(_args(), 1, 2) == 0
    assert capsys.readouterr().out == ""


def test_reference_arm_without_binary(monkeypatch, capsys):
    monkeypatch.setattr(bench, "REF_BIN", ROOT / "oracle" / "_ref" / "no_such_binary")
    assert bench.run_reference(_args(), 0, 1) == 0
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference" and line["unavailable"]


@pytest.mark.skipif(not bench.REF_BIN.exists(), reason="reference CLI not built (oracle/_ref)")
def test_reference_run_summary_parse():
    trials, elapsed, iters = bench._run_ref(0.04, 50, 4, 7, True, 5)
    assert trials == 4 and elapsed >= 0.0 and 4 <= iters <= 4 * 50


class _FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _smi(sm, reasons=()):
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    flags = ["Active" if n in reasons else "Not Active" for n in names]
    return ", ".join(["0", str(sm), "1965", "950.00", "0x0000000000000000"] + flags)


def test_clock_record_counts_only_the_timed_region():
    s = bench.ClockSampler(0)
    s.proc = _FakeProc()
    s.lines = [_smi(1200, ("hw_slowdown",))]                        # warm-up: not part of the record
    s.mark()
    s.lines += [_smi(1965), _smi(1965, ("sw_power_cap",)), _smi(1950)]
    rec = s.stop()
    assert rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"] and rec["samples"] == 3


def test_clock_record_without_nvidia_smi():
    rec = bench.ClockSampler(0).stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]


def test_package_wilson_interval_matches_reference_cli():
    """The interval the bench reports beside its failure counts is the reference's Wilson
    interval (jointbp_ets.cpp:4388-4399): equal, to the CLI's 8 printed decimals, on every
    golden run summary; clipped to [0, 1]; none for no trials."""
    from conftest import GOLDEN
    from joint_bp_plus_pp_b200 import wilson_interval
    cli = json.loads((GOLDEN / "cli_summaries.json").read_text())
    assert cli
    for name, c in cli.items():
        s = c["summary"]
        lo, hi = wilson_interval(int(s["trials"]), int(s["failures"]))
        assert "[" + f"{lo:.8f},{hi:.8f}" + "]" == s["ci95"].replace(" ", ""), name
    assert wilson_interval(0, 0) is None
    lo, hi = wilson_interval(655360, 0)
    assert lo == 0.0 and 5.8e-6 < hi < 5.9e-6
    lo, hi = wilson_interval(40, 40)
    assert hi == 1.0 and 0.9 < lo < 1.0
