"""The FP64 bit-exact kernels normalize with one reciprocal per divisor instead of four
divisions (recip_for_div / div_by_recip in joint_bp_plus_pp_b200/csrc/kernels_bp.cuh,
Markstein's FMA-based division).  This test compiles the same sequence for the host and checks
it against IEEE division on random and edge-case pairs of the guarded domain; the GPU parity
tests then check the kernels bit for bit against the reference's decisions."""
import subprocess
from pathlib import Path

import pytest

SRC = Path(__file__).resolve().parent / "native" / "reciprocal_division_check.c"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = tmp_path_factory.mktemp("div") / "check"
    r = subprocess.run(["gcc", "-O2", "-mfma", "-o", str(exe), str(SRC), "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip(f"no host compiler with FMA: {r.stderr[:200]}")
    return exe


@pytest.mark.parametrize("lo,hi", [(-960, 900), (-905, -880), (880, 905), (-1022, -890)])
def test_reciprocal_division_equals_ieee_division(checker, lo, hi):
    r = subprocess.run([str(checker), "4000000", str(lo), str(hi)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert "mismatches 0" in r.stdout
