"""CPU restatement of the learned sector map's network (float64 numpy).

TEST INFRASTRUCTURE ONLY: the checker for pyffa_b200.learned and the
ffa_mlp_* entry points (imported by tests/ only).

The network has no counterpart in the reference (PyFFA tracks with the
pushers only); what it learns is the one-sector map of the azimuth-domain
tracker that follows FunctionForSEO (src/FFAG_track.py:1597-1640).

Residual MLP y = x + x Ws + bs + q(x) Wq + f(x) (q: the 15 products
x_i x_j, i <= j < 5), f = L4 . SiLU . L3 . SiLU . L2 .
SiLU . L1, layer widths 6 -> 256 -> 256 -> 256 -> 6 (W_l: (n_in, n_out),
L(h) = h W_l + b_l), loss = mean over samples and the first `n_fit` outputs
of (y - target)^2.

`bf16=True` rounds the operands of the tensor-core products to bfloat16
(round to nearest even) the way the GPU kernels stage them: both factors of
every product except layer 1, where only W1 is rounded (the kernels keep the
float32 input exact: training multiplies it in float32, inference splits it
into high and low bfloat16 parts against a doubled W1); the
products themselves, biases, SiLU, the skip layer and the loss stay in
float64 here (float32 on the GPU).  The GPU evaluates SiLU(z) as
h + h tanh(h), h = z / 2, with the hardware tanh approximation (relative
error below 2^-10.9); here it is exact.  With bf16 the GPU results agree to
that and to float32 accumulation; without it, to bfloat16 rounding error.
"""
from __future__ import annotations

import numpy as np

FITTED_SHAPES = {"W1": (6, 256), "b1": (256,), "W2": (256, 256), "b2": (256,), "W3": (256, 256),
                 "b3": (256,), "W4": (256, 6), "b4": (6,), "Ws": (6, 6), "bs": (6,), "Wq": (15, 6)}
QUAD = [(i, j) for i in range(5) for j in range(i, 5)]


def quad(x):
    """The 15 second-order skip features s_i s_j, i <= j < 5."""
    return np.stack([x[:, i] * x[:, j] for i, j in QUAD], 1)


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _mm(a, b, round_):
    return (bf16(a) @ bf16(b)) if round_ else (a @ b)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, x, bf16_ops=False):
    """params: dict with FITTED_SHAPES; x (B, 6).  Returns (y, cache)."""
    x = np.asarray(x, np.float64)
    h = x
    cache = {"h0": x}
    for l in (1, 2, 3):
        if l == 1:
            # the input stays exact (the kernels split it into two bfloat16
            # parts); only W1 is rounded
            z = h @ (bf16(params["W1"]) if bf16_ops else params["W1"]) + params["b1"]
        else:
            z = _mm(h, params[f"W{l}"], bf16_ops) + params[f"b{l}"]
        cache[f"z{l}"] = z
        h = silu(z)
        cache[f"h{l}"] = h
    f = _mm(h, params["W4"], bf16_ops) + params["b4"]
    cache["f"] = f
    y = x + x @ params["Ws"] + params["bs"] + quad(x) @ params["Wq"] + f
    return y, cache


def loss_and_grads(params, x, target, n_fit=4, bf16_ops=False):
    """Mean squared error over the first n_fit outputs and its gradients
    (every parameter; the entries of unfitted outputs are zero)."""
    y, c = forward(params, x, bf16_ops)
    B = x.shape[0]
    d = np.zeros_like(y)
    d[:, :n_fit] = 2.0 * (y[:, :n_fit] - target[:, :n_fit]) / (B * n_fit)
    sse = float(np.sum((y[:, :n_fit] - target[:, :n_fit]) ** 2))
    g = {"Ws": np.asarray(x, np.float64).T @ d, "bs": d.sum(0), "Wq": quad(np.asarray(x, np.float64)).T @ d,
         "W4": _mm(c["h3"].T, d, bf16_ops), "b4": d.sum(0)}
    dh = _mm(d, params["W4"].T, bf16_ops)
    for l in (3, 2, 1):
        dz = dh * dsilu(c[f"z{l}"])
        g[f"W{l}"] = _mm(c[f"h{l - 1}"].T, dz, bf16_ops)
        g[f"b{l}"] = dz.sum(0)
        if l > 1:
            dh = _mm(dz, params[f"W{l}"].T, bf16_ops)
    return sse, g


def adam(params, grads, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, frozen=()):
    """One Adam step in place (bias-corrected), skipping the `frozen` names."""
    c1, c2 = 1 - beta1 ** step, 1 - beta2 ** step
    for k in params:
        if k in frozen:
            continue
        m[k] = beta1 * m[k] + (1 - beta1) * grads[k]
        v[k] = beta2 * v[k] + (1 - beta2) * grads[k] ** 2
        params[k] = params[k] - lr * (m[k] / c1) / (np.sqrt(v[k] / c2) + eps)


def apply_map(params, s, n_apply, radius2=0.0, bf16_ops=True):
    """n_apply applications of the map to normalised states s (B, 6):
    columns 0..3 advance, e and the spare column stay; a state outside the
    domain (u^2 + pu^2 > radius2, v^2 + pv^2 > radius2 or |e| > 1, checked
    before each application when radius2 > 0) stops.  Returns (s, applied)."""
    s = np.array(s, np.float64)
    applied = np.zeros(len(s), np.int64)
    act = np.ones(len(s), bool)
    for _ in range(n_apply):
        if radius2 > 0:
            inside = ((s[:, 0] ** 2 + s[:, 1] ** 2 <= radius2) & (s[:, 2] ** 2 + s[:, 3] ** 2 <= radius2)
                      & (np.abs(s[:, 4]) <= 1.0))
            act &= inside
        y, _ = forward(params, s, bf16_ops)
        s[act, :4] = y[act, :4]
        applied += act
    return s, applied
