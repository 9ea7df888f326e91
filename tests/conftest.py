"""Shared pytest configuration: the `gpu` marker and fixture helpers."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

TESTS = Path(__file__).resolve().parent
ROOT = TESTS.parent
GOLDEN = TESTS / "golden"
sys.path.insert(0, str(TESTS))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def load_sim_case(name):
    meta = json.loads((GOLDEN / f"sim_{name}.json").read_text())
    vec = np.load(GOLDEN / f"vec_{name}.npz")
    return meta, vec["err"], vec["est"]


SIM_CASE_NAMES = sorted(p.name[4:-5] for p in GOLDEN.glob("sim_*.json"))


@pytest.fixture(scope="session")
def oracle():
    from oracle_bind import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def decoder():
    from joint_bp_plus_pp_b200 import Decoder
    return Decoder.from_params()
