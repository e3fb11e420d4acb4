"""Turn-by-turn diagnostics of tracked bunches: states where particles cross
one azimuth (from crossing records), the errors of one run against another
at that azimuth, FFT tunes and rms emittances.

The tune estimator restates the reference's FFT tune analysis
(tune_from_xpx and parabolic_interpolate, benchmarks/Benchmark_SC_kvTune.py:
318-365): the turn-by-turn signal x - i px / s (s = std(px) / std(x)), mean
removed, zero-padded FFT, DC bin ignored, the magnitude peak refined by a
parabola through it and its two neighbours.  The reference forms x + i px / s,
whose peak sits at 1 - Q for a betatron rotation (px lagging x by a quarter
period); the conjugate signal puts it at the fractional tune Q itself.  The rms emittance is
FFAG_Emit's sqrt(<x^2><x'^2> - <x x'>^2) (src/FFAG_Emit.py:9-18).
"""
from __future__ import annotations

import numpy as np

C_LIGHT = 2.99792458e8


def _speed(post: np.ndarray, solver: str, E0_J: float | None) -> np.ndarray:
    """Particle speed from post-step record columns (r, vr, z, vz, fi, f5):
    f5 is dfi/dt for Boris, the total energy [J] for RK4."""
    if solver == "RK4":
        g = post[:, 5] / E0_J
        return C_LIGHT * np.sqrt(1.0 - 1.0 / (g * g))
    return np.sqrt(post[:, 1] ** 2 + post[:, 3] ** 2 + (post[:, 0] * post[:, 5]) ** 2)


def crossing_table(rec: np.ndarray, n: int, dt: float, solver: str = "Boris", E0_J: float | None = None):
    """All crossings of records `rec` (rows of 23: target, particle, step,
    ratio, pre r vr z vz fi f5 rf, post ..., flags, fields; a 24th column,
    where present, is the step's end time) as a per-particle turn-by-turn
    table (turns, n, 6): r, vr, z, vz interpolated to the azimuth, the speed,
    and the crossing time (from the step's end time, or (step + ratio) dt
    without it); NaN where a particle has fewer crossings than the
    most-crossing one."""
    rec = np.asarray(rec)
    idx = rec[:, 1].astype(np.int64)
    order = np.lexsort((rec[:, 2], idx))
    rec, idx = rec[order], idx[order]
    counts = np.bincount(idx, minlength=n)
    turns = int(counts.max()) if counts.size else 0
    out = np.full((turns, n, 6), np.nan)
    if turns == 0:
        return out
    first = np.concatenate([[0], np.cumsum(counts)[:-1]])
    k = np.arange(rec.shape[0]) - first[idx]
    a = rec[:, 3:4]
    pre, post = rec[:, 4:11], rec[:, 11:18]
    x = pre + a * (post - pre)
    out[k, idx, 0:4] = x[:, 0:4]
    out[k, idx, 4] = _speed(post, solver, E0_J)
    if rec.shape[1] > 23:
        out[k, idx, 5] = rec[:, 23] - dt + rec[:, 3] * dt
    else:
        out[k, idx, 5] = (rec[:, 2] + rec[:, 3]) * dt
    return out


def at_azimuth(rec: np.ndarray, n: int, dt: float, solver: str = "Boris", E0_J: float | None = None) -> np.ndarray:
    """The last crossing of each particle (n, 6), NaN where it has none."""
    tab = crossing_table(rec, n, dt, solver, E0_J)
    out = np.full((n, 6), np.nan)
    for t in range(tab.shape[0]):
        ok = np.isfinite(tab[t, :, 0])
        out[ok] = tab[t, ok]
    return out


def _emittance(x, xp):
    x = x - x.mean()
    xp = xp - xp.mean()
    return float(np.sqrt(max(0.0, np.mean(x * x) * np.mean(xp * xp) - np.mean(x * xp) ** 2)))


def azimuth_errors(ref: np.ndarray, got: np.ndarray) -> dict:
    """Errors of `got` against `ref` (rows of at_azimuth) over the particles
    both have: radius |dr|/r (max and median), arrival time |dt|/t, momentum
    |dp|/p, vr, z, vz relative to their amplitude, rms emittances."""
    ok = np.isfinite(ref[:, 0]) & np.isfinite(got[:, 0])
    a, b = ref[ok], got[ok]
    g = lambda v: 1.0 / np.sqrt(1.0 - (v / C_LIGHT) ** 2)
    pa, pb = g(a[:, 4]) * a[:, 4], g(b[:, 4]) * b[:, 4]
    dr = np.abs(b[:, 0] - a[:, 0]) / a[:, 0]
    e = {"n": int(ok.sum()), "r": float(dr.max()), "r_median": float(np.median(dr)),
         "t": float(np.max(np.abs(b[:, 5] - a[:, 5]) / a[:, 5])),
         "p": float(np.max(np.abs(pb - pa) / pa))}
    for name, col in (("vr", 1), ("z", 2), ("vz", 3)):
        e[name + "_amp"] = float(np.abs(b[:, col] - a[:, col]).max() / np.abs(a[:, col]).max())
    for name, (cx, cv) in (("emit_x", (0, 1)), ("emit_z", (2, 3))):
        ea = _emittance(a[:, cx], a[:, cv] / a[:, 4])
        eb = _emittance(b[:, cx], b[:, cv] / b[:, 4])
        e[name] = float(abs(eb - ea) / ea)
    return e


def _parabolic_peak(amp: np.ndarray, k: int) -> float:
    y0, y1, y2 = amp[k - 1], amp[k], amp[k + 1]
    den = y0 - 2.0 * y1 + y2
    return float(k) if den == 0 else k + 0.5 * (y0 - y2) / den


def fft_tune(x: np.ndarray, px: np.ndarray, pad_factor: int = 4) -> float:
    """Fractional tune in [0, 1) of one turn-by-turn signal (x, px)."""
    x = np.asarray(x, np.float64)
    px = np.asarray(px, np.float64)
    if x.size != px.size or x.size < 8:
        raise ValueError("x and px need the same length, at least 8 turns")
    sx, sp = x.std(), px.std()
    scale = sp / sx if sx > 0 and sp > 0 else 1.0
    zz = x - 1j * (px / scale)
    zz = zz - zz.mean()
    nfft = int(pad_factor * x.size)
    mag = np.abs(np.fft.fft(zz, n=nfft))
    mag[0] = 0.0
    k = min(max(int(np.argmax(mag)), 1), nfft - 2)
    return (_parabolic_peak(mag, k) % nfft) / nfft


def tunes(table: np.ndarray) -> np.ndarray:
    """Horizontal and vertical fractional tunes (n, 2) from a crossing table
    (turns, n, 6); NaN for particles with a gap in their record."""
    n = table.shape[1]
    out = np.full((n, 2), np.nan)
    for i in range(n):
        col = table[:, i, :]
        if not np.isfinite(col[:, 0]).all():
            continue
        out[i, 0] = fft_tune(col[:, 0], col[:, 1])
        out[i, 1] = fft_tune(col[:, 2], col[:, 3])
    return out
