"""GPU tests of the learned flip proposal: the training kernels' gradients and the BF16
tensor-core inference against the CPU oracle (oracle/mlp_oracle.py), stall-state collection,
training, and what the trained network gains over the decoder without it."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def rand_problem(n, seed):
    rng = np.random.default_rng(seed)
    params = rng.normal(0, 0.25, mlp_oracle.NPARAMS).astype(np.float32)
    x = rng.normal(0, 1, (n, 8)).astype(np.float32)
    y = (rng.random((n, 2)) < 0.2).astype(np.float32)
    return params, x, y


@pytest.mark.parametrize("n", [1, 37, 1000, 20000])
def test_gpu_gradient_matches_oracle(decoder, n):
    """FP32 forward/backward kernels against the FP64 oracle (relative to the gradient's scale)."""
    params, x, y = rand_problem(n, n)
    g, loss = decoder.mlp_grad(params, x, y, pos_weight=3.0)
    lref, gref = mlp_oracle.loss_and_grad(params, x, y, pos_weight=3.0)
    assert abs(loss - lref) <= 1e-4 * abs(lref) + 1e-6
    scale = np.abs(gref).max()
    assert np.abs(g - gref).max() <= 2e-4 * scale, np.abs(g - gref).max() / scale


def test_gpu_bf16_inference_matches_oracle(decoder):
    params, x, _ = rand_problem(5003, 11)          # not a multiple of the 16-row tile
    out = decoder.mlp_infer(params, x)
    ref = mlp_oracle.infer_bf16(params, x)
    exact = mlp_oracle.loss_and_grad  # noqa: F841  (FP64 forward is the training reference)
    err = np.abs(out - ref)
    assert err.max() <= 2e-2 * (1 + np.abs(ref).max()), err.max()
    confident = np.abs(ref) > 0.05
    assert (np.sign(out[confident]) == np.sign(ref[confident])).mean() > 0.999


def test_gpu_training_reduces_loss(decoder):
    """A separable synthetic task: Adam on the GPU drives the loss well below its start."""
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (40000, 8)).astype(np.float32)
    y = np.stack([(x[:, 0] + 0.5 * x[:, 6] > 0.8), (x[:, 2] - x[:, 7] > 1.0)], 1).astype(np.float32)
    from joint_bp_plus_pp_b200 import mlp_init
    p0 = mlp_init(1)
    _, l0 = decoder.mlp_grad(p0, x, y)
    p1, hist = decoder.mlp_train(p0, x, y, epochs=6, batch=2048, lr=3e-3)
    _, l1 = decoder.mlp_grad(p1, x, y)
    assert l1 < 0.3 * l0 and hist[-1] < hist[0]


def test_collect_stall_states(decoder):
    from joint_bp_plus_pp_b200 import Options
    o = Options(precision="fp16", engine="resident", max_iter=60, enable_pp=True, learned_from=6)
    x, y, st = decoder.collect_stall_states(77, 4000, 0.05, o, 200000)
    assert st["trials"] == 4000 and len(x) > 0
    assert np.isfinite(x).all() and (x[:, :4] <= 0).all() and (x[:, :4] >= -4).all()
    assert ((x[:, 4:6] >= 0) & (x[:, 4:6] <= 1)).all() and ((x[:, 6:] >= 0) & (x[:, 6:] <= 1)).all()
    assert set(np.unique(y)) <= {0.0, 1.0} and y.sum() > 0
    # the collection does not change the decoding beyond the decision-history bits kept in the
    # low mantissa bits of the variable totals (a 2^-17 relative perturbation)
    st2, _ = decoder.simulate(77, 4000, 0.05, Options(precision="fp16", engine="resident", max_iter=60,
                                                       enable_pp=True))
    assert st2["failures"] == st["failures"]
    assert abs(st2["total_iters"] - st["total_iters"]) <= 1e-3 * st2["total_iters"]


def test_learned_needs_a_model(decoder):
    from joint_bp_plus_pp_b200 import JbpError, Options
    decoder.set_flip_model(None)
    with pytest.raises(JbpError):
        decoder.simulate(1, 8, 0.05, Options(precision="fp16", engine="resident", max_iter=30, enable_pp=True,
                                             learned_from=10))


@pytest.mark.parametrize("prec", ["fp16", "fp32"])
def test_trained_model_gain(decoder, prec):
    """The shipped model (trained by joint_bp_plus_pp_b200.learned on the decoder's own stalled
    states) against the same decoder without it, on the same 40,000 trials at p=0.045 (max-iter
    300, post-processing on, proposals from iteration 6).  What the network gains: trials that
    stall are ended at the stall by an exactly syndrome-matching correction instead of BP
    iterating on, so their iteration counts drop, their outcomes are not worse, and the logical
    error rate of the whole run is not worse within its 95% interval."""
    from joint_bp_plus_pp_b200 import Options, load_flip_model, wilson_interval
    params = load_flip_model()
    assert params is not None, "data/flip_mlp_params.npy missing"
    decoder.set_flip_model(params)
    N = 40000
    base = dict(precision=prec, engine="resident", max_iter=300, enable_pp=True)
    s0, r0 = decoder.simulate(606, N, 0.045, Options(**base))
    s1, r1 = decoder.simulate(606, N, 0.045, Options(learned_from=6, **base))
    decoder.set_flip_model(None)
    acc = (r1["ets_used_flags"] & 32) != 0
    assert s1["learned_attempts"] > 0 and acc.sum() > 0
    assert acc.sum() >= 0.7 * s1["learned_attempts"]            # most proposals are accepted
    assert r1["syndrome_ok"][acc].all()                          # only exact syndrome matches
    assert r1["success"][acc].sum() >= r0["success"][acc].sum()  # the same trials, not worse
    assert r1["iterations"][acc].mean() < r0["iterations"][acc].mean()
    # the run's total: the accepted trials' savings are of the order of the perturbation the
    # learned instantiation's decision-history bits bring to the others (2^-17 of |A|), so the
    # total is bounded by that perturbation rather than required to fall
    assert s1["total_iters"] <= s0["total_iters"] * (1 + 1e-3)
    lo0, hi0 = wilson_interval(N, s0["failures"])
    assert s1["failures"] / N <= hi0, (s1["failures"], s0["failures"])
