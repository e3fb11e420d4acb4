"""Oracle of the GPU bunch generator (test infrastructure; only tests/ may
import it).

A numpy restatement of ffa_bunch_sample: Philox4x32-10 (Salmon, Moraes,
Dror and Shaw, SC 2011; multipliers 0xD2511F53 / 0xCD9E8D57, key increments
0x9E3779B9 / 0xBB67AE85, ten rounds), uniforms (x + 1/2) 2^-32, Box-Muller
normals, the distribution shapes of src/FFAG_Distribution.py:76-1149 with
their emittance factors, the Twiss transformation of TwissContainer
(src/FFAG_Distribution.py:16-73) and the p-format row of
GenerateInitDistributionDtInjNew (:1152-1345).  The draw layout (counter
words: particle id low and high, draw group, sub-bunch; rejection attempts
in groups 2a, 2a + 1; the longitudinal plane from group 2^30) is the one
ffa_bunch_sample documents, so rows agree with the GPU's to rounding.
"""
from __future__ import annotations

import numpy as np

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)
MAX_ATTEMPTS = 64
GAUSS, KV, WATERBAG, HOLLOW, UNIFORM_GAUSS = 0, 1, 2, 3, 4
LONG_GROUP = 1 << 30


def philox4x32_10(c0, c1, c2, c3, key):
    """Vectorised Philox4x32-10: four uint32 arrays (as uint64) -> four."""
    c = [np.asarray(x, np.uint64) & MASK for x in (c0, c1, c2, c3)]
    k0, k1 = np.uint64(key & 0xFFFFFFFF), np.uint64((key >> 32) & 0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c = [(hi1 ^ c[1] ^ k0) & MASK, lo1, (hi0 ^ c[3] ^ k1) & MASK, lo0]
        k0 = np.uint64((int(k0) + W0) & 0xFFFFFFFF)
        k1 = np.uint64((int(k1) + W1) & 0xFFFFFFFF)
    return c


def uniforms(ids, group, sub, seed):
    ids = np.asarray(ids, np.uint64)
    out = philox4x32_10(ids & MASK, ids >> np.uint64(32), np.full_like(ids, group), np.full_like(ids, sub), seed)
    return [(x.astype(np.float64) + 0.5) * 2.0 ** -32 for x in out]


def box_muller(u1, u2):
    rad = np.sqrt(-2.0 * np.log(u1))
    return rad * np.cos(2 * np.pi * u2), rad * np.sin(2 * np.pi * u2)


def kv1d(ua, ub):
    x = np.sin(2 * np.pi * (ua - 0.5))
    return x, np.where(ub < 0.5, -1.0, 1.0) * np.sqrt(1.0 - x * x)


def _twiss(t, scale):
    a, b, e = t[0], t[1], t[2] * scale
    return np.sqrt(b * e), np.sqrt(e / b), a


def sample(n, seed, sub, transverse, longitudinal, twiss, centre, fi, bunch_id, cut_off=-1.0,
           uniform_length=0.0, uniform_sigma=0.0, id0=0):
    """n p-format rows as ffa_bunch_sample writes them."""
    ids = np.arange(id0, id0 + n, dtype=np.uint64)
    ts = {KV: 4.0, WATERBAG: 6.0}.get(transverse, 1.0)
    ls = {KV: 2.0, WATERBAG: 4.0}.get(longitudinal, 1.0)
    if transverse in (KV, WATERBAG):
        u = uniforms(ids, 0, sub, seed)
        rho = np.sqrt(u[1])
        xn, yn = rho * np.cos(2 * np.pi * (u[0] - 0.5)), rho * np.sin(2 * np.pi * (u[0] - 0.5))
        p0 = np.sqrt(np.abs(1.0 - rho * rho))
        xpn, ypn = p0 * np.cos(2 * np.pi * (u[2] - 0.5)), p0 * np.sin(2 * np.pi * (u[2] - 0.5))
        if transverse == WATERBAG:
            g = np.sqrt(np.sqrt(u[3]))
            xn, xpn, yn, ypn = g * xn, g * xpn, g * yn, g * ypn
    elif transverse == HOLLOW:
        done = np.zeros(n, bool)
        xn = xpn = yn = ypn = np.zeros(n)
        for a in range(MAX_ATTEMPTS):
            u = uniforms(ids, 2 * a, sub, seed)
            w = uniforms(ids, 2 * a + 1, sub, seed)
            x1, x1p = kv1d(u[0], u[1])
            y1, y1p = kv1d(u[2], u[3])
            gx, gy = 0.4 + 0.6 * w[0], 0.4 + 0.6 * w[1]
            q = (gx * x1) ** 2 + (gy * y1) ** 2
            take = ~done
            xn, xpn = np.where(take, gx * x1, xn), np.where(take, gx * x1p, xpn)
            yn, ypn = np.where(take, gy * y1, yn), np.where(take, gy * y1p, ypn)
            done |= take & (q >= 0.3) & (q <= 1.0)
            if done.all():
                break
    else:
        okx, oky = np.zeros(n, bool), np.zeros(n, bool)
        xn = xpn = yn = ypn = np.zeros(n)
        for a in range(MAX_ATTEMPTS):
            u = uniforms(ids, 2 * a, sub, seed)
            n0, n1 = box_muller(u[0], u[1])
            n2, n3 = box_muller(u[2], u[3])
            xn, xpn = np.where(okx, xn, n0), np.where(okx, xpn, n1)
            yn, ypn = np.where(oky, yn, n2), np.where(oky, ypn, n3)
            okx |= (cut_off <= 0) | (n0 * n0 + n1 * n1 <= cut_off * cut_off)
            oky |= (cut_off <= 0) | (n2 * n2 + n3 * n3 <= cut_off * cut_off)
            if okx.all() and oky.all():
                break
    um, uc, ua = _twiss(twiss[0], ts)
    x, xp = um * xn, uc * (xpn - ua * xn)
    um, uc, ua = _twiss(twiss[1], ts)
    y, yp = um * yn, uc * (ypn - ua * yn)
    if longitudinal == UNIFORM_GAUSS:
        u = uniforms(ids, LONG_GROUP, sub, seed)
        n0, _ = box_muller(u[1], u[2])
        t, dE = uniform_length * (u[0] - 0.5), uniform_sigma * n0
    else:
        if longitudinal in (KV, WATERBAG, HOLLOW):
            u = uniforms(ids, LONG_GROUP, sub, seed)
            tn, en = kv1d(u[0], u[1])
            if longitudinal == WATERBAG:
                g = np.sqrt(u[2])
                tn, en = g * tn, g * en
            elif longitudinal == HOLLOW:
                g = 0.4 + 0.6 * u[2]
                tn, en = g * tn, g * en
        else:
            ok = np.zeros(n, bool)
            tn = en = np.zeros(n)
            for a in range(MAX_ATTEMPTS):
                u = uniforms(ids, LONG_GROUP + a, sub, seed)
                a0, a1 = box_muller(u[0], u[1])
                tn, en = np.where(ok, tn, a0), np.where(ok, en, a1)
                ok |= (cut_off <= 0) | (a0 * a0 + a1 * a1 <= cut_off * cut_off)
                if ok.all():
                    break
        um, uc, ua = _twiss(twiss[2], ls)
        t, dE = um * tn, uc * (en - ua * tn)
    out = np.zeros((n, 16))
    out[:, 0], out[:, 1], out[:, 2], out[:, 3] = x + centre[0], xp + centre[1], y + centre[2], yp + centre[3]
    out[:, 4] = fi
    out[:, 5] = dE + centre[4]
    out[:, 6] = t + centre[5]
    out[:, 13] = bunch_id
    out[:, 14] = out[:, 15] = ids.astype(np.float64)
    return out
