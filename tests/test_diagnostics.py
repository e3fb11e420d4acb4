"""Turn-by-turn diagnostics on the host: the FFT tune estimator against known
rotations, and the crossing-record tables built from synthetic records."""
import numpy as np

from pyffa_b200 import diagnostics as D


def test_fft_tune_recovers_rotation_tunes():
    rng = np.random.default_rng(0)
    t = np.arange(1000)
    for q in (0.137, 0.5951, 0.7813, 0.93):
        x = 2e-3 * np.cos(2 * np.pi * q * t + 0.3)
        px = -5e3 * np.sin(2 * np.pi * q * t + 0.3)
        got = D.fft_tune(x + 1e-9 * rng.standard_normal(t.size), px)
        assert abs(got - q) < 2e-4, (q, got)


def test_crossing_table_orders_turns_and_interpolates():
    n, turns, dt = 3, 4, 1e-9
    rows = []
    for i in range(n):
        for k in range(turns):
            if i == 2 and k == 3:
                continue              # particle 2 is lost before its last crossing
            pre = np.array([8.0 + k, 1.0 + i * i, 0.01 * (1 + i), 2.0 - i * i, 1.0, 2e7, 0.0])
            post = pre + np.array([0.2, 0.4, 0.002, 0.0, 0.01, 0.0, 0.0])
            rows.append(np.concatenate([[0, i, 100 * k + i, 0.25], pre, post, [1, 1, 0, 0, 0]]))
    rec = np.array(rows)[::-1]         # any order in, sorted per particle and step out
    tab = D.crossing_table(rec, n, dt)
    assert tab.shape == (turns, n, 6)
    assert np.allclose(tab[:, 0, 0], 8.05 + np.arange(turns))
    assert np.isnan(tab[3, 2, 0]) and np.isfinite(tab[2, 2, 0])
    assert np.allclose(tab[1, 1, 5], (101 + 0.25) * dt)
    last = D.at_azimuth(rec, n, dt)
    assert np.allclose(last[:, 0], [11.05, 11.05, 10.05])
    e = D.azimuth_errors(last, last)
    assert e["r"] == 0.0 and e["p"] == 0.0 and e["n"] == n
