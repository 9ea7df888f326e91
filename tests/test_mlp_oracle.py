"""CPU checks of the MLP oracle itself (finite differences), so that it can judge the GPU kernels."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle  # noqa: E402


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    params = rng.normal(0, 0.3, mlp_oracle.NPARAMS)
    x = rng.normal(0, 1, (40, 8))
    y = (rng.random((40, 2)) < 0.3).astype(float)
    loss, g = mlp_oracle.loss_and_grad(params, x, y, pos_weight=3.0)
    for i in rng.choice(mlp_oracle.NPARAMS, 60, replace=False):
        e = np.zeros_like(params)
        e[i] = 1e-6
        fd = (mlp_oracle.loss_and_grad(params + e, x, y, 3.0)[0] - mlp_oracle.loss_and_grad(params - e, x, y, 3.0)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])


def test_oracle_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], np.float32)
    r = mlp_oracle.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[4] == 0.0
    assert abs(r[3] + 3.140625) < 1e-6
