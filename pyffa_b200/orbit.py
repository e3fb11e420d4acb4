"""Closed orbits, tunes and closed-orbit tables of the mid-plane field.

Host-side (float64, numpy) counterpart of the reference's closed-orbit search
(FFAG_SearchSEO, src/FFAG_track.py:1142-1586): the reference integrates the
orbit with theta as the independent variable and Newton-iterates the
one-sector map for (r, pr); tunes come from the trace of the one-sector
transfer matrix, Q = N acos(tr/2) / (2 pi) (src/FFAG_track.py:1325-1371).
Here every energy of a scan is integrated at once (vectorised RK4 in theta)
and the linearised vertical motion is carried along for the vertical tune.

Equations (mid-plane field Bz = B0 r^k F(theta), proton charge q > 0, the
pushers' sign convention B_eff = -B):
    dr/dtheta  = r p_r / p_theta
    dp_r/dtheta = p_theta - q r Bz
    dz/dtheta  = r p_z / p_theta
    dp_z/dtheta = -q r (p_r / p_theta * B_theta - B_r),  B_r = dBz/dr z, B_theta = dBz/dtheta z / r
"""
from __future__ import annotations

import numpy as np

from .constants import Q
from .fields import convex_params


class MidplaneField:
    def __init__(self, cfg: dict):
        bm = cfg["Bmap"]
        self.B0, self.k = bm["coefficients_tupel"]
        self.cp = convex_params(bm)
        self.N = bm["NSector"]
        self.P = 2 * np.pi / self.N
        if bm.get("SpiralAngle_deg", 0) != 0:
            raise NotImplementedError("this helper (synthetic inputs) takes a zero spiral angle; "
                                      "spiral lattices: pyffa_b200.seo.FFAG_SearchSEO")

    def flutter(self, th):
        th = th - self.P * np.floor(th / self.P)
        f = np.zeros_like(th)
        fp = np.zeros_like(th)
        with np.errstate(over="ignore"):
            for x0, x1, W0, y01, y02 in self.cp:
                ks = 16.0 / W0
                y = y02 * abs(y01)
                s1 = 1 / (1 + np.exp(-ks * (th - x0)))
                s2 = 1 / (1 + np.exp(ks * (th - x1)))
                f += y * s1 * s2
                fp += y * (ks * s1 * (1 - s1) * s2 - s1 * ks * s2 * (1 - s2))
        return f, fp

    def __call__(self, r, th):
        f, fp = self.flutter(np.broadcast_to(th, np.shape(r)).astype(np.float64))
        brk = self.B0 * r ** self.k
        return brk * f, self.B0 * self.k * r ** (self.k - 1) * f, brk * fp


def _rhs(th, y, p, fld):
    r, pr, z, pz = y
    pth = np.sqrt(p * p - pr * pr - pz * pz)
    Bz, dBr, dBt = fld(r, th)
    Br = dBr * z
    Bt = dBt / r * z
    return np.stack([r * pr / pth, pth - Q * r * Bz, r * pz / pth, -Q * r * (pr / pth * Bt - Br)])


def track_sector(y0, p, fld, nstep=2000, th0=0.0, record=False):
    """RK4 in theta over one sector for states y0 (4, M); returns the end
    state (and the recorded (r, pr/p_theta, ds/dtheta) along the way)."""
    h = fld.P / nstep
    y = np.array(y0, dtype=np.float64)
    th = th0
    rec = []
    for _ in range(nstep):
        if record:
            rec.append(y.copy())
        k1 = _rhs(th, y, p, fld)
        k2 = _rhs(th + h / 2, y + h / 2 * k1, p, fld)
        k3 = _rhs(th + h / 2, y + h / 2 * k2, p, fld)
        k4 = _rhs(th + h, y + h * k3, p, fld)
        y = y + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        th += h
    if record:
        rec.append(y.copy())
        return y, np.array(rec)
    return y


def closed_orbits(cfg: dict, Ek_MeV, r_guess=None, nstep=2000, tol=1e-12, max_iter=30):
    """Closed orbit (r, p_r/p_theta) at theta = 0 and the tunes for each
    energy.  Returns dict of arrays r0, pr0, Qx, Qz, trx, trz."""
    from .synthetic import momentum, orbit_radius
    fld = MidplaneField(cfg)
    E = np.atleast_1d(np.asarray(Ek_MeV, dtype=np.float64))
    p = momentum(E)
    r = np.asarray(r_guess, np.float64) * np.ones_like(E) if r_guess is not None else orbit_radius(E) * 0.96
    pr = np.zeros_like(E)
    M = E.size
    d_r, d_p = 1e-7, 1e-7
    for _ in range(max_iter):
        # 5 probes per energy: base, dr, dpr, dz, dpz
        y0 = np.zeros((4, M, 5))
        y0[0] = r[:, None]
        y0[1] = pr[:, None]
        y0[0, :, 1] += d_r
        y0[1, :, 2] += d_p * p
        y0[2, :, 3] = d_r
        y0[3, :, 4] = d_p * p
        pp = np.repeat(p[:, None], 5, axis=1)
        out = track_sector(y0.reshape(4, -1), pp.reshape(-1), fld, nstep).reshape(4, M, 5)
        f0 = np.stack([out[0, :, 0] - r, out[1, :, 0] - pr])
        Mx = np.empty((M, 2, 2))
        Mx[:, :, 0] = ((out[:2, :, 1] - out[:2, :, 0]) / d_r).T
        Mx[:, :, 1] = ((out[:2, :, 2] - out[:2, :, 0]) / (d_p * p)).T
        Mz = np.empty((M, 2, 2))
        Mz[:, :, 0] = ((out[2:, :, 3] - out[2:, :, 0]) / d_r).T
        Mz[:, :, 1] = ((out[2:, :, 4] - out[2:, :, 0]) / (d_p * p)).T
        A = Mx - np.eye(2)[None]
        dx = np.linalg.solve(A, -f0.T[..., None])[..., 0]
        r = r + dx[:, 0]
        pr = pr + dx[:, 1]
        if np.all(np.abs(dx[:, 0]) < tol * np.abs(r)):
            break
    trx = 0.5 * (Mx[:, 0, 0] + Mx[:, 1, 1])
    trz = 0.5 * (Mz[:, 0, 0] + Mz[:, 1, 1])
    with np.errstate(invalid="ignore"):
        Qx = np.where(np.abs(trx) < 1, np.arccos(np.clip(trx, -1, 1)) / (2 * np.pi) * fld.N, np.nan)
        Qz = np.where(np.abs(trz) < 1, np.arccos(np.clip(trz, -1, 1)) / (2 * np.pi) * fld.N, np.nan)
    pth = np.sqrt(p * p - pr * pr)
    return {"Ek": E, "r0": r, "pr0": pr / pth, "p_r": pr, "Qx": Qx, "Qz": Qz, "trx": trx, "trz": trz}


def seo_tables(cfg: dict, Ek_axis, nfi=361, nstep=2000):
    """Closed-orbit tables on a uniform fi axis over [0, 2 pi]:
    r0(Ek, fi), pr0(Ek, fi) = p_r/p_theta and the orbit length per turn
    (the inputs of the space-charge step, src/FFAG_Bunch.py:1227-1287)."""
    fld = MidplaneField(cfg)
    co = closed_orbits(cfg, Ek_axis, nstep=nstep)
    from .synthetic import momentum
    E = co["Ek"]
    p = momentum(E)
    y0 = np.stack([co["r0"], co["p_r"], np.zeros_like(E), np.zeros_like(E)])
    _, rec = track_sector(y0, p, fld, nstep, record=True)   # rec (nstep+1, 4, M)
    th_s = np.linspace(0.0, fld.P, nstep + 1)
    r_s = rec[:, 0, :]
    pr_s = rec[:, 1, :] / np.sqrt(p ** 2 - rec[:, 1, :] ** 2)
    fi_axis = np.linspace(0.0, 2 * np.pi, nfi)
    fm = fi_axis - fld.P * np.floor(fi_axis / fld.P)
    r_tab = np.stack([np.interp(fm, th_s, r_s[:, m]) for m in range(E.size)])
    pr_tab = np.stack([np.interp(fm, th_s, pr_s[:, m]) for m in range(E.size)])
    drdth = r_s * pr_s
    ds = np.sqrt(r_s ** 2 + drdth ** 2)
    perim = fld.N * np.trapezoid(ds, th_s, axis=0)
    return {"Ek_axis": E, "fi_axis": fi_axis, "r": r_tab, "pr": pr_tab, "perimeter": perim,
            "Qx": co["Qx"], "Qz": co["Qz"]}
