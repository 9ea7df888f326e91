"""CPU oracle of the learned flip proposal's MLP (test infrastructure only).

The MLP has no counterpart in the reference; this numpy restatement is the checker of the
library's GPU kernels: FP64 forward/backward of the loss (gradients of jbp_mlp_grad) and the
BF16-operand / FP32-accumulate forward of the tensor-core inference (jbp_mlp_infer and the
decoder's fused proposal).  Parameter layout: W1[64][8], b1[64], W2[64][64], b2[64],
W3[2][64], b3[2].
"""
import numpy as np

SHAPES = [("W1", (64, 8)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (2, 64)), ("b3", (2,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(params):
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def softplus(z):
    return np.where(z > 0, z + np.log1p(np.exp(-np.abs(z))), np.log1p(np.exp(z)))


def loss_and_grad(params, x, y, pos_weight=1.0):
    """Mean over samples of sum_o [pw*y*softplus(-z) + (1-y)*softplus(z)] and its gradient."""
    p = unpack(params)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(x)
    a1 = x @ p["W1"].T + p["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(a2, 0)
    z = h2 @ p["W3"].T + p["b3"]
    loss = (pos_weight * y * softplus(-z) + (1 - y) * softplus(z)).sum() / n
    s = 1 / (1 + np.exp(-z))
    dz = (pos_weight * y * (s - 1) + (1 - y) * s) / n
    g = {"W3": dz.T @ h2, "b3": dz.sum(0)}
    dh2 = (dz @ p["W3"]) * (a2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ p["W2"]) * (a1 > 0)
    g["W1"] = dh1.T @ x
    g["b1"] = dh1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SHAPES])


def bf16(a):
    """Round to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def infer_bf16(params, x):
    """Logits with BF16 inputs, weights and hidden activations, FP32 accumulation and biases."""
    p = unpack(params)
    h = bf16(x).astype(np.float32)
    h = bf16(np.maximum(h @ bf16(p["W1"]).T.astype(np.float32) + p["b1"].astype(np.float32), 0))
    h = bf16(np.maximum(h @ bf16(p["W2"]).T.astype(np.float32) + p["b2"].astype(np.float32), 0))
    return h @ bf16(p["W3"]).T.astype(np.float32) + p["b3"].astype(np.float32)
