"""Batched orbit scan, host side (no GPU): crossing records of known
one-turn maps, shuffled and split over two launches, are paired turn to turn
and fitted back to their fixed points and tunes."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from pyffa_b200 import coscan  # noqa: E402


def _map(q, beta, alpha):
    mu = 2 * math.pi * q
    g = (1 + alpha * alpha) / beta
    c, s = math.cos(mu), math.sin(mu)
    return np.array([[c + alpha * s, beta * s], [-g * s, c - alpha * s]])


def test_records_fit_back_to_fixed_points_and_tunes():
    rng = np.random.default_rng(1)
    counts = [1, 3, 17]
    tunes = [(0.5951, 0.7813), (0.31, 0.12), (0.87, 0.44)]
    # physical scales: positions ~ 8.5 m and mm offsets, velocities ~ 1e8 m/s
    # and 1e4 m/s offsets (the fit has to rescale them to stay conditioned)
    unit = np.array([1e-3, 2e5, 1e-3, 2e5])
    fixed = np.array([8.5, 2e7, 0.0, 0.0]) + rng.normal(0, 1, (3, 4)) * unit
    guess = fixed + rng.normal(0, 0.1, (3, 4)) * unit
    inst = np.repeat(np.arange(3), counts)
    N, T = len(inst), 40
    rec, ratio = [], 0.3
    state = fixed[inst] + rng.normal(0, 0.5, (N, 4)) * unit
    Ms = [[_map(qx, 2e-8, 0.4), _map(qz, 11e-8, -1.3)] for qx, qz in tunes]
    for t in range(T):
        for pidx in range(N):
            x = state[pidx]
            d = rng.normal(0, 0.1, 4) * unit
            row = np.zeros(23)
            row[1], row[2], row[3] = pidx, 100 * t + pidx % 7, ratio
            row[4:8] = x - ratio * d
            row[11:15] = x + (1 - ratio) * d
            rec.append(row)
        for pidx in range(N):
            i = inst[pidx]
            for pl in (0, 1):
                sl = slice(2 * pl, 2 * pl + 2)
                state[pidx, sl] = Ms[i][pl] @ (state[pidx, sl] - fixed[i, sl]) + fixed[i, sl]
    rec = np.array(rec)
    f64 = dict(dtype=torch.float64)
    S = torch.zeros((2, 3, 3, 3), **f64)
    Y = torch.zeros((2, 3, 2, 3), **f64)
    cr = torch.zeros(3, **f64)
    last = torch.zeros((N, 4), **f64)
    has = torch.zeros(N, dtype=torch.bool)
    gv = torch.as_tensor(guess)
    it = torch.as_tensor(inst)
    # two launches (turns 0..17 and 18..39), each in shuffled order
    for part in (rec[rec[:, 2] < 1800], rec[rec[:, 2] >= 1800]):
        part = torch.as_tensor(part[rng.permutation(len(part))])
        x = part[:, 4:8] + part[:, 3:4] * (part[:, 11:15] - part[:, 4:8])
        coscan.accumulate_crossings(part[:, 1].long(), part[:, 2].long(), x, gv, it, 100 * T, last, has, S, Y, cr,
                                    torch.as_tensor(np.tile(1.0 / unit, (3, 1))))
    fix, q, good = coscan.fit_one_turn(S.numpy(), Y.numpy())
    assert good.all()
    assert np.allclose(guess + fix * unit, fixed, atol=0, rtol=1e-12)
    assert np.all(np.abs(guess + fix * unit - fixed) <= 1e-9 * unit)
    assert np.allclose(q, np.array(tunes), atol=1e-10)
    assert cr.numpy().tolist() == [c * T for c in counts]


def test_instance_counts_log_uniform():
    c = coscan.instance_counts(256, 4096, seed=0)
    assert c.min() >= 1 and c.max() <= 4096 and len(c) == 256
    assert 300 < c.mean() < 700


def _record(pre, post):
    row = np.zeros(23)
    row[4:10], row[11:17] = pre, post
    return row


def test_crossing_states_exact_on_straight_lines():
    """A drift crossing azimuth 0 at any point of the step: r, vr, z, vz of
    the crossing come out exact (a linear interpolation in the azimuth
    misses r by up to r'' dphi^2 / 8)."""
    dt = 3.7e-10
    rng = np.random.default_rng(5)
    rows, want = [], []
    for frac in rng.uniform(0.01, 0.99, 50):
        # straight line through (8.13 m, 0) at the crossing, 6.7 deg off the tangent
        v, a = 1.9e8, 0.1171
        vx, vy, vz = v * math.sin(a), v * math.cos(a), 2e5
        X, Yc, Zc = 8.13 + rng.normal(0, 1e-3), 0.0, rng.normal(0, 1e-3)
        def polar(t):
            x, y, z = X + vx * t, Yc + vy * t, Zc + vz * t
            r, fi = math.hypot(x, y), math.atan2(y, x)
            vr = (x * vx + y * vy) / r
            f5 = (x * vy - y * vx) / (r * r)
            return [r, vr, z, vz, fi % (2 * math.pi), f5]
        rows.append(_record(polar(-frac * dt), polar((1 - frac) * dt)))
        want.append([X, vx, Zc, vz])
    rec = torch.as_tensor(np.array(rows))
    got = coscan.crossing_states(rec, dt).numpy()
    want = np.array(want)
    assert np.abs(got[:, 0] - want[:, 0]).max() < 1e-12
    assert np.abs(got[:, 2] - want[:, 2]).max() < 1e-12
    assert np.abs(got[:, 1] / want[:, 1] - 1).max() < 1e-10
    # the azimuth-linear interpolation of r is off by tens of micrometres here
    lin = rec[:, 4] + (rec[:, 11] - rec[:, 4]) * (-(rec[:, 8] - 2 * math.pi * (rec[:, 8] > 3)) /
                                                  (rec[:, 15] - rec[:, 8] + 2 * math.pi * (rec[:, 8] > 3)))
    assert np.abs(lin.numpy() - want[:, 0]).max() > 1e-5


def test_launch_steps_persistent_and_memory_bound(monkeypatch):
    """One launch per iteration when the records fit half the free device
    memory (with 3x for the accumulation), else the longest launch that
    does; persistent=False keeps the 5-records-per-particle launches."""
    import torch
    from pyffa_b200 import _lib

    class Cap:                       # a CrossingCapture's sizing fields
        def __init__(self, n, dt, f_max):
            self.bunch = type("B", (), {"n": n})()
            self.x = type("X", (), {"ntargets": 1})()
            self.dt, self.f_max = dt, f_max

        def max_steps(self):
            return max(1, int(3 * 2 * np.pi / (self.dt * self.f_max)))

    def need(cap, L):
        per = 2 + int(np.ceil(L * cap.dt * cap.f_max / (2 * np.pi)))
        return 4 * cap.bunch.n * per * 8 * _lib.CROSSING_RECORD

    cap = Cap(162321, 8.2e-11, 3.79e7)
    scan = object.__new__(coscan.BatchedOrbitScan)
    scan.dev, scan.steps = "cuda:0", 666804
    scan.persistent = True
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (180 << 30, 180 << 30))
    assert scan._launch_steps(cap) == scan.steps                       # 180 GB free: one launch
    free = 2 * need(cap, 100000)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (free, free))
    L = scan._launch_steps(cap)
    assert cap.max_steps() < L < scan.steps
    assert need(cap, L) <= free // 2 < need(cap, L + 1)                # the longest that fits
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (0, 0))
    assert scan._launch_steps(cap) == cap.max_steps()                  # nothing free: the short launches
    scan.persistent = False
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda dev=None: (180 << 30, 180 << 30))
    assert scan._launch_steps(cap) == cap.max_steps()


def test_fixed_shape_accumulation_equals_direct():
    """The graph mode's fixed-shape accumulation (whole record buffer, rows
    past the count sent to a dummy particle and instance) gives the direct
    accumulation's sums, pairs and last states, whatever the stale rows hold
    (NaN included), over two launches in shuffled order."""
    rng = np.random.default_rng(5)
    f64 = dict(dtype=torch.float64)
    I, counts = 3, [2, 5, 4]
    inst = np.repeat(np.arange(I), counts)
    N, turns, dt = len(inst), 6, 2e-10
    rows = []
    for t in range(turns):
        for p in range(N):
            r = 8.5 + 1e-3 * rng.standard_normal()
            f5 = 2.3e7 / r                       # rad/s
            row = np.zeros(23)
            row[1], row[2] = p, 3000 * t + 17 * p
            d0 = rng.uniform(0.1, 0.9) * f5 * dt  # the step crosses azimuth 0
            for o, fi in ((4, -d0), (11, f5 * dt - d0)):
                row[o:o + 6] = [r + 1e-6 * rng.standard_normal(), 1e4 * rng.standard_normal(),
                                1e-3 * rng.standard_normal(), 1e4 * rng.standard_normal(), fi, f5]
            rows.append(row)
    rec = np.array(rows)
    launches = [rec[rec[:, 2] < 3000 * 3], rec[rec[:, 2] >= 3000 * 3]]
    scale = torch.as_tensor(np.vstack([np.tile([1e3, 1e-4, 1e3, 1e-4], (I, 1)), np.ones((1, 4))]))
    gv = torch.zeros((I + 1, 4), **f64)
    gv[:I, 0] = 8.5
    inst_ext = torch.as_tensor(np.concatenate([inst, [I]]))

    def state(n_inst, n_part):
        return (torch.zeros((2, n_inst, 3, 3), **f64), torch.zeros((2, n_inst, 2, 3), **f64),
                torch.zeros(n_inst, **f64), torch.zeros((n_part, 4), **f64),
                torch.zeros(n_part, dtype=torch.bool))
    S1, Y1, c1, last1, has1 = state(I, N)
    S2, Y2, c2, last2, has2 = state(I + 1, N + 1)
    C = max(len(x) for x in launches) + 7
    for part in launches:
        part = part[rng.permutation(len(part))]
        pt = torch.as_tensor(part)
        coscan.accumulate_crossings(pt[:, 1].long(), pt[:, 2].long(), coscan.crossing_states(pt, dt),
                                    gv[:I], inst_ext[:N], 3000 * turns, last1, has1, S1, Y1, c1, scale[:I])
        buf = rng.standard_normal((C, 23))           # stale rows past the count
        buf[len(part):len(part) + 3] = np.nan
        buf[:len(part)] = part
        coscan.accumulate_crossings_fixed(torch.as_tensor(buf), torch.tensor(len(part)), dt, gv, inst_ext,
                                          3000 * turns, last2, has2, S2, Y2, c2, scale)
    assert torch.allclose(S2[:, :I], S1, rtol=1e-13, atol=0) and torch.allclose(Y2[:, :I], Y1, rtol=1e-13, atol=0)
    assert torch.equal(c2[:I], c1) and c1.tolist() == [float(turns * c) for c in counts]
    assert torch.equal(has2[:N], has1) and bool(has1.all())
    assert torch.allclose(last2[:N], last1, rtol=1e-15, atol=0)
    # (turns - 1) pairs per particle in the normal equations' constant term
    assert S1[0, :, 2, 2].tolist() == [float((turns - 1) * c) for c in counts]


def test_fit_sums_layout_unpacks_to_normal_equations():
    """The per-instance sums in the layout the push kernel accumulates
    (ffa_crossing.fit_sums: per plane f0 f0, f0 f1, f0, f1 f1, f1, 1, then
    u'_0 f0, u'_0 f1, u'_0, u'_1 f0, u'_1 f1, u'_1; the crossing count last)
    unpack to the S, Y and counts of accumulate_crossings for the same
    crossings."""
    from pyffa_b200 import _lib
    rng = np.random.default_rng(9)
    I, counts, turns = 3, [2, 5, 4], 7
    inst = np.repeat(np.arange(I), counts)
    N = len(inst)
    u = rng.standard_normal((turns, N, 4))          # scaled crossing states, turn by turn
    sums = np.zeros((I, _lib.FIT_SUMS))
    for t in range(turns):
        for p in range(N):
            k = inst[p]
            if t > 0:
                for pl in (0, 1):
                    f0, f1 = u[t - 1, p, 2 * pl], u[t - 1, p, 2 * pl + 1]
                    a, b = u[t, p, 2 * pl], u[t, p, 2 * pl + 1]
                    sums[k, 12 * pl:12 * pl + 12] += [f0 * f0, f0 * f1, f0, f1 * f1, f1, 1.0,
                                                      a * f0, a * f1, a, b * f0, b * f1, b]
            sums[k, 24] += 1.0
    S, Y, c = coscan.unpack_fit_sums(sums)
    f64 = dict(dtype=torch.float64)
    S1, Y1, c1 = torch.zeros((2, I, 3, 3), **f64), torch.zeros((2, I, 2, 3), **f64), torch.zeros(I, **f64)
    last, has = torch.zeros((N, 4), **f64), torch.zeros(N, dtype=torch.bool)
    p = torch.as_tensor(np.tile(np.arange(N), turns))
    step = torch.as_tensor(np.repeat(np.arange(turns), N) * 1000)
    coscan.accumulate_crossings(p, step, torch.as_tensor(u.reshape(-1, 4)), torch.zeros((I, 4), **f64),
                                torch.as_tensor(inst), 1000 * turns, last, has, S1, Y1, c1)
    np.testing.assert_allclose(S, S1.numpy(), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(Y, Y1.numpy(), rtol=1e-13, atol=1e-13)
    np.testing.assert_array_equal(c, c1.numpy())
    assert np.array_equal(S, S.transpose(0, 1, 3, 2))
