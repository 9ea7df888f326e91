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


RCP_SRC = Path(__file__).resolve().parent / "native" / "reciprocal_rn_check.c"


@pytest.fixture(scope="module")
def rcp_checker(tmp_path_factory):
    exe = tmp_path_factory.mktemp("rcp") / "check"
    r = subprocess.run(["gcc", "-O2", "-mfma", "-o", str(exe), str(RCP_SRC), "-lm"], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip(f"no host compiler with FMA: {r.stderr[:200]}")
    return exe


@pytest.mark.parametrize("lo,hi", [(-900, 899), (-900, -890), (890, 899), (-2, 2)])
def test_branch_free_reciprocal_equals_ieee_division(rcp_checker, lo, hi):
    """recip_rn_fast's sequence (two Newton steps, then the exact-remainder choice among y and
    its neighbours), started from approximations with relative errors up to 2^-16 (the hardware
    approximation it starts from on the device is within 2^-19.9), gives the correctly rounded
    1/s over the fast path's whole domain."""
    r = subprocess.run([str(rcp_checker), "3000000", str(lo), str(hi)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert "mismatches 0" in r.stdout


@pytest.mark.gpu
def test_device_reciprocal_equals_division():
    """The same sequence on the GPU, from the hardware approximation, against the correctly
    rounded division intrinsic on 10^9 divisors."""
    from joint_bp_plus_pp_b200 import check_reciprocal
    bad, first = check_reciprocal(10 ** 9, seed=12345)
    assert bad == 0, (bad, first)
