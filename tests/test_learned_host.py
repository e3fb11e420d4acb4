"""Learned sector map, host side (no GPU): the oracle network pinned by
finite differences, its bfloat16 rounding against torch's, the parameter
layout shared with libffa_cuda.so, and the tune / emittance diagnostics."""
import math

import numpy as np
import pytest

from oracle import mlp as M
from pyffa_b200 import _lib, learned


def _params(seed, scale_out=0.05):
    rng = np.random.default_rng(seed)
    d = learned.to_dict(learned.init_params(seed))
    d["W4"] = rng.standard_normal(d["W4"].shape) * scale_out / 16
    for k in ("b1", "b2", "b3"):
        d[k] = 0.1 * rng.standard_normal(d[k].shape)
    d["b4"] = 0.01 * rng.standard_normal(6)
    d["Ws"] = 0.1 * rng.standard_normal((6, 6))
    d["bs"] = 0.01 * rng.standard_normal(6)
    d["Wq"] = 0.05 * rng.standard_normal((15, 6))
    return d


def test_layout_matches_header():
    assert learned.N_PARAMS == _lib.MLP_PARAMS
    assert sum(int(np.prod(sh)) for _, sh in learned.LAYOUT.values()) == _lib.MLP_PARAMS
    d = _params(1)
    d2 = learned.to_dict(learned.from_dict(d))
    for k in d:
        assert np.array_equal(d2[k], d[k].astype(np.float32).astype(np.float64))
    p = learned.from_dict(d)
    # padding stays zero: rows 6.. of W1, columns 6, 7 of W4
    assert not learned.block(p, "W1")[6:].any() and not learned.block(p, "W4")[:, 6:].any()


def test_oracle_gradients_match_finite_differences():
    d = _params(2)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (24, 6))
    x[:, 5] = 0
    t = rng.uniform(-1, 1, (24, 6))
    sse, g = M.loss_and_grads(d, x, t, n_fit=4)
    n = 24 * 4

    def loss(p):
        return M.loss_and_grads(p, x, t, n_fit=4)[0] / n
    for name, idx in (("W1", (2, 17)), ("b1", (5,)), ("W2", (100, 3)), ("b2", (77,)), ("W3", (9, 250)),
                      ("b3", (0,)), ("W4", (31, 2)), ("b4", (3,)), ("Ws", (4, 1)), ("bs", (0,)), ("Wq", (7, 2))):
        h = 1e-6
        p1 = {k: v.copy() for k, v in d.items()}
        p2 = {k: v.copy() for k, v in d.items()}
        p1[name][idx] += h
        p2[name][idx] -= h
        fd = (loss(p1) - loss(p2)) / (2 * h)
        assert abs(fd - g[name][idx]) <= 1e-7 + 1e-5 * abs(fd), (name, fd, g[name][idx])
    # outputs that are not fitted get no gradient
    assert not g["b4"][4:].any() and not g["W4"][:, 4:].any()


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    a = np.concatenate([rng.standard_normal(20000) * 10.0 ** rng.integers(-8, 8, 20000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 65504.0]]).astype(np.float32)
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(a), ref)


def test_oracle_bf16_forward_close_to_float64():
    d = _params(5)
    x = np.random.default_rng(6).uniform(-1, 1, (64, 6))
    y64, c64 = M.forward(d, x)
    y16, c16 = M.forward(d, x, bf16_ops=True)
    f = np.abs(c64["f"]).max()
    assert np.abs(c16["f"] - c64["f"]).max() <= 2e-2 * f


def test_apply_map_domain_rule():
    d = _params(7)
    s = np.zeros((4, 6))
    s[0, :4] = [0.1, 0.2, 0.0, 0.1]
    s[1, :4] = [1.2, 0.0, 0.0, 0.0]      # outside in x
    s[2, 4] = 1.5                         # outside in energy
    s[3, :4] = [0.5, 0.5, 0.5, 0.5]
    out, applied = M.apply_map(d, s, 3, radius2=1.0)
    assert applied.tolist()[1:3] == [0, 0]
    assert np.array_equal(out[1], s[1]) and np.array_equal(out[2], s[2])
    assert applied[0] >= 1 and applied[3] >= 1


def test_adam_matches_formula():
    p = {"a": np.array([1.0, -2.0])}
    g = {"a": np.array([0.5, -0.25])}
    m = {"a": np.zeros(2)}
    v = {"a": np.zeros(2)}
    M.adam(p, g, m, v, 1, 0.1)
    # first bias-corrected step moves each entry by lr * sign(g)
    assert np.allclose(p["a"], [0.9, -1.9], atol=1e-7)


def test_tunes_from_rotation_record():
    T, n = 400, 5
    q = np.array([0.6031, 0.2217])
    rng = np.random.default_rng(8)
    amp = rng.uniform(0.1, 1.0, (n, 2))
    ph = rng.uniform(0, 2 * np.pi, (n, 2))
    rec = np.zeros((T + 1, n, 4))
    k = np.arange(T + 1)[:, None]
    for j, pl in ((0, 0), (2, 1)):
        ang = ph[None, :, pl] + 2 * np.pi * q[pl] * k
        # X - i PX advances by +mu: X = A cos(ang), PX = -A sin(ang)
        rec[:, :, j] = amp[:, pl] * np.cos(ang)
        rec[:, :, j + 1] = -amp[:, pl] * np.sin(ang)
    t = learned.tunes(rec)
    assert np.allclose(t, q[None, :], atol=1e-12)


def test_rms_emittance_of_gaussian():
    rng = np.random.default_rng(9)
    n = 200000
    a = np.zeros((n, 4))
    a[:, 0] = 8.5 + 2e-3 * rng.standard_normal(n)
    a[:, 1] = 1e-3 * rng.standard_normal(n)
    a[:, 2] = 1e-3 * rng.standard_normal(n)
    a[:, 3] = 0.5e-3 * rng.standard_normal(n)
    e = learned.rms_emittance(a)
    assert abs(e[0] / 2e-6 - 1) < 0.01 and abs(e[1] / 0.5e-6 - 1) < 0.01


def test_sample_domain_uniform_in_disc():
    s = learned.sample_domain(100000, np.random.default_rng(10), radius=1.0)
    for j in (0, 2):
        r2 = s[:, j] ** 2 + s[:, j + 1] ** 2
        assert r2.max() <= 1.0
        # uniform in the disc: r^2 is uniform on [0, 1]
        assert abs(np.mean(r2) - 0.5) < 0.01
    assert s[:, 4].min() >= -1 and s[:, 4].max() <= 1


def test_lr_schedule_cosine_with_warmup():
    total, lr, lr_min, warmup = 1000, 2e-3, 1e-5, 200
    s = learned.lr_schedule(total, lr, lr_min, warmup)
    assert s.shape == (total,)
    for k in (0, 1, 199, 200, 500, 999):
        ref = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * k / total))
        if k < warmup:
            ref *= (k + 1) / warmup
        assert abs(s[k] - ref) <= 1e-15 * lr
    assert s[warmup - 1] > s[0] and np.all(np.diff(s[warmup:]) < 0)
    assert s.min() > 0
