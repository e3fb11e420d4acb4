"""Injected-bunch generation (GenerateBunches and its helpers,
src/FFAG_Distribution.py:16-1640), seeded.

The reference draws every particle from Python's and NumPy's global random
streams one particle at a time (unseeded), so its bunches are reproducible
only by pre-generating them.  Here each generator draws all particles of a
sub-bunch at once from a numpy Generator (seeded through ``BunchPara["Seed"]``
or the ``rng`` argument); the transformations — normalised coordinates to
(u, u') through the Twiss parameters, the KV / water-bag / Gauss / hollow
shapes and their emittance factors, the injection point on the closed orbit
from the SEO tables, the painting offsets — are the reference's, so the
bunches agree with the reference's in distribution (moments, emittances,
Twiss), not particle by particle.

The output is the reference's p-format matrix (N x 16: r, pr, z, pz, fi,
Ek [MeV], inj_t [ns], flags 0, RF phase 0, space-charge fields 0, Bunch_ID,
Local_ID, Global_ID), one block per painted sub-bunch.
"""
from __future__ import annotations

import math
import os
import re

import numpy as np

from .constants import COLUMNS

# ---------------------------------------------------------------- Twiss


class TwissContainer:
    """alpha, beta, emittance; (u_norm, u'_norm) -> (u, u')
    (src/FFAG_Distribution.py:16-73)."""

    def __init__(self, alpha, beta, emittance):
        self.alpha = alpha
        self.beta = beta
        self.emittance = emittance
        self._init()

    def _init(self):
        self.gamma = (1.0 + self.alpha ** 2) / self.beta
        self.u_max = math.sqrt(self.beta * self.emittance)
        self.up_coeff = math.sqrt(self.emittance / self.beta)
        self.up_max = math.sqrt(self.gamma * self.emittance)

    def setEmittance(self, emittance):
        self.emittance = emittance
        self._init()

    def getNormalizedH(self, u, up):
        return (u ** 2 + (self.alpha * u + self.beta * up) ** 2) / (self.beta * self.emittance)

    def getU_Max(self):
        return self.u_max

    def getUP_Max(self):
        return self.up_max

    def getU_UP(self, u_norm, up_norm):
        return self.u_max * u_norm, self.up_coeff * (up_norm - self.alpha * u_norm)

    def getAlphaBetaGammaEmitt(self):
        return self.alpha, self.beta, self.gamma, self.emittance

    def getAlphaBetaEmitt(self):
        return self.alpha, self.beta, self.emittance


_default_rng = np.random.default_rng()


class _Dist:
    """sample(n, rng) draws n particles at once; getCoordinates() draws one."""

    def getCoordinates(self):
        return tuple(float(c[0]) for c in self.sample(1, _default_rng))


class KVDist1D(_Dist):
    """1D KV; 100 % emittance = 2 x rms."""

    def __init__(self, twiss=None):
        twiss = twiss or TwissContainer(0., 1., 1.)
        a, b, e = twiss.getAlphaBetaEmitt()
        self.twiss = TwissContainer(a, b, 2 * e)

    def sample(self, n, rng):
        x = np.sin(2 * np.pi * (rng.random(n) - 0.5))
        xp = rng.choice((-1.0, 1.0), n) * np.sqrt(1.0 - x ** 2)
        return self.twiss.getU_UP(x, xp)

    def getTwissContainers(self):
        return (self.twiss,)


class WaterBagDist1D(_Dist):
    def __init__(self, twiss=None):
        twiss = twiss or TwissContainer(0., 1., 1.)
        a, b, e = twiss.getAlphaBetaEmitt()
        self.kv = KVDist1D(TwissContainer(a, b, 2 * e))

    def sample(self, n, rng):
        u, up = self.kv.sample(n, rng)
        g = np.sqrt(rng.random(n))
        return g * u, g * up

    def getTwissContainers(self):
        return self.kv.getTwissContainers()


class HollowWaterBagDist1D(_Dist):
    def __init__(self, twiss=None):
        twiss = twiss or TwissContainer(0., 1., 1.)
        a, b, e = twiss.getAlphaBetaEmitt()
        self.kv = KVDist1D(TwissContainer(a, b, e / 2))

    def sample(self, n, rng):
        u, up = self.kv.sample(n, rng)
        g = rng.uniform(0.4, 1.0, n)
        return g * u, g * up

    def getTwissContainers(self):
        return self.kv.getTwissContainers()


class GaussDist1D(_Dist):
    def __init__(self, twiss=None, cut_off=-1.0):
        self.twiss = twiss or TwissContainer(0., 1., 1.)
        self.cut_off = cut_off

    def sample(self, n, rng):
        x = rng.standard_normal(n)
        xp = rng.standard_normal(n)
        if self.cut_off > 0:
            bad = x ** 2 + xp ** 2 > self.cut_off ** 2
            while bad.any():
                k = int(bad.sum())
                x[bad], xp[bad] = rng.standard_normal(k), rng.standard_normal(k)
                bad = x ** 2 + xp ** 2 > self.cut_off ** 2
        return self.twiss.getU_UP(x, xp)

    def getTwissContainers(self):
        return (self.twiss,)


class KVDist2D(_Dist):
    """2D KV (uniform on the 4D hyper-ellipsoid surface); 100 % = 4 x rms."""

    def __init__(self, twissX=None, twissY=None):
        twissX = twissX or TwissContainer(0., 1., 1.)
        twissY = twissY or TwissContainer(0., 1., 1.)
        ax, bx, ex = twissX.getAlphaBetaEmitt()
        ay, by, ey = twissY.getAlphaBetaEmitt()
        self.twissX = TwissContainer(ax, bx, 4 * ex)
        self.twissY = TwissContainer(ay, by, 4 * ey)

    def sample(self, n, rng):
        phi = 2 * np.pi * (rng.random(n) - 0.5)
        rho = np.sqrt(rng.random(n))
        x, y = rho * np.cos(phi), rho * np.sin(phi)
        p0 = np.sqrt(np.abs(1.0 - rho ** 2))
        phi = 2 * np.pi * (rng.random(n) - 0.5)
        xp, yp = p0 * np.cos(phi), p0 * np.sin(phi)
        return (*self.twissX.getU_UP(x, xp), *self.twissY.getU_UP(y, yp))

    def getTwissContainers(self):
        return self.twissX, self.twissY


class WaterBagDist2D(_Dist):
    def __init__(self, twissX=None, twissY=None):
        twissX = twissX or TwissContainer(0., 1., 1.)
        twissY = twissY or TwissContainer(0., 1., 1.)
        ax, bx, ex = twissX.getAlphaBetaEmitt()
        ay, by, ey = twissY.getAlphaBetaEmitt()
        self.kv = KVDist2D(TwissContainer(ax, bx, 6.0 * ex / 4.0), TwissContainer(ay, by, 6.0 * ey / 4.0))

    def sample(self, n, rng):
        x, xp, y, yp = self.kv.sample(n, rng)
        g = np.sqrt(np.sqrt(rng.random(n)))
        return g * x, g * xp, g * y, g * yp

    def getTwissContainers(self):
        return self.kv.getTwissContainers()


class GaussDist2D(_Dist):
    def __init__(self, twissX=None, twissY=None, cut_off=-1.0):
        self.gx = GaussDist1D(twissX, cut_off)
        self.gy = GaussDist1D(twissY, cut_off)

    def sample(self, n, rng):
        return (*self.gx.sample(n, rng), *self.gy.sample(n, rng))

    def getTwissContainers(self):
        return self.gx.twiss, self.gy.twiss


class IndependentHollowWaterBagDist2D(_Dist):
    """Hollow water bags in x-x' and y-y', kept where 0.3 <= (x/xm)^2 + (y/ym)^2 <= 1."""

    def __init__(self, twissX=None, twissY=None):
        self.hx = HollowWaterBagDist1D(twissX)
        self.hy = HollowWaterBagDist1D(twissY)

    def sample(self, n, rng):
        out = [np.zeros(n) for _ in range(4)]
        todo = np.arange(n)
        xm, ym = self.hx.kv.twiss.getU_Max(), self.hy.kv.twiss.getU_Max()
        while todo.size:
            x, xp = self.hx.sample(todo.size, rng)
            y, yp = self.hy.sample(todo.size, rng)
            q = x ** 2 / xm ** 2 + y ** 2 / ym ** 2
            ok = (q >= 0.3) & (q <= 1)
            for o, v in zip(out, (x, xp, y, yp)):
                o[todo[ok]] = v[ok]
            todo = todo[~ok]
        return tuple(out)

    def getTwissContainers(self):
        return self.hx.getTwissContainers(), self.hy.getTwissContainers()


class CustomDist3D(_Dist):
    """Transverse 2D distribution times a longitudinal 1D one."""

    def __init__(self, dist_transverse, dist_longitudinal):
        self.dist_transverse = dist_transverse
        self.dist_longitudinal = dist_longitudinal

    def sample(self, n, rng):
        return (*self.dist_transverse.sample(n, rng), *self.dist_longitudinal.sample(n, rng))

    def getTwissContainers(self):
        return tuple(self.dist_transverse.getTwissContainers()) + (self.dist_longitudinal.getTwissContainers(),)


def create_distribution(dist_type, twiss_transverse=None, twiss_longitudinal=None):
    """src/FFAG_Distribution.py:1107-1149."""
    if dist_type == "gauss":
        return GaussDist2D(*twiss_transverse) if twiss_transverse is not None else GaussDist1D(twiss_longitudinal)
    if dist_type == "kv":
        return KVDist2D(*twiss_transverse) if twiss_transverse is not None else KVDist1D(twiss_longitudinal)
    if dist_type == "waterbag":
        return WaterBagDist2D(*twiss_transverse) if twiss_transverse is not None else \
            WaterBagDist1D(twiss_longitudinal)
    if dist_type == "hollow_waterbag":
        return IndependentHollowWaterBagDist2D(*twiss_transverse) if twiss_transverse is not None else \
            HollowWaterBagDist1D(twiss_longitudinal)
    if dist_type in ("match", "UniformGauss"):
        return GaussDist1D(twiss_longitudinal)
    raise ValueError(f"Unknown distribution type: {dist_type}")


# ------------------------------------------------------ SEO table lookups


def _four_points(X, xi):
    """find_four_points_non_uniform_vector (src/FFAG_MathTools.py:109-145)."""
    right = np.searchsorted(X, xi, side="right")
    left = right - 1
    idx = np.stack([left - 1, left, right, right + 1])
    lo = (left - 1) < 0
    idx[:, lo] = np.array([0, 1, 2, 3])[:, None]
    hi = (right + 1) > len(X) - 1
    idx[:, hi] = np.array([len(X) - 4, len(X) - 3, len(X) - 2, len(X) - 1])[:, None]
    return idx


def Lagrange_interp_2D_vect(X, Y, Z, Xi, Yi):
    """Four-by-four-point Lagrange interpolation (src/FFAG_MathTools.py:274-315);
    returns (values, out-of-range flags)."""
    X, Y, Z = np.asarray(X), np.asarray(Y), np.asarray(Z)
    Xi, Yi = np.atleast_1d(Xi).astype(np.float64), np.atleast_1d(Yi).astype(np.float64)
    ix, iy = _four_points(X, Xi), _four_points(Y, Yi)
    xs, ys = X[ix], Y[iy]

    def weights(s, v):
        L = np.zeros((4, len(v)))
        for a in range(4):
            o = [b for b in range(4) if b != a]
            num = (v - s[o[0]]) * (v - s[o[1]]) * (v - s[o[2]])
            L[a] = num / (s[a] - s[o[0]]) / (s[a] - s[o[1]]) / (s[a] - s[o[2]])
        return L

    Lx, Ly = weights(xs, Xi), weights(ys, Yi)
    zs = Z[ix[:, None, :], iy[None, :, :]]
    val = np.sum(Lx[:, None, :] * Ly[None, :, :] * zs, axis=(0, 1))
    flag = (np.searchsorted(X, Xi, side="right") - 2 < 0) | (np.searchsorted(X, Xi, side="right") + 1 > len(X) - 1)
    return val, flag


def LoadSEOBetaFunc(SEOPATHName, Ek_c, fi_c):
    """(beta_z, beta_r, alpha_z, alpha_r) at (Ek_c, fi_c) from the Twiss files
    (src/FFAG_Distribution.py:1430-1457).  As in the reference, fi_c [rad] is
    reduced modulo the table's azimuth span converted to rad but looked up on
    the table's azimuth axis, which is in degrees."""
    out = []
    for name in ("BetaFuncZ.txt", "BetaFuncR.txt", "AlphaFuncZ.txt", "AlphaFuncR.txt"):
        d = np.loadtxt(os.path.join(SEOPATHName, name), skiprows=1)
        Ek_axis, fi_axis, M = d[1:, 0], d[0, 1:], d[1:, 1:]
        fi = np.mod(np.array([fi_c]), np.deg2rad(fi_axis[-1] - fi_axis[0]))
        out.append(Lagrange_interp_2D_vect(Ek_axis, fi_axis, M, np.array([Ek_c]), fi)[0][0])
    return tuple(out)


def _segments(points):
    """Polyline points (n, 2) -> segments (n - 1, 4) = x1, y1, x2, y2
    (CentralLine2Segments, src/FFAG_Utils.py:278-286)."""
    p = np.asarray(points, np.float64)
    return np.column_stack([p[:-1], p[1:]])


def _segment_crossings(A, B):
    """Every segment of A against every segment of B (FindIntersectionVect,
    src/FFAG_Utils.py:32-152): the crossing flags (a, b) -- bounding boxes
    overlap and each segment's ends lie strictly on both sides of the other's
    line -- and the signed distances of A's two ends from B's line (a, b)."""
    A = np.atleast_2d(A)[:, None, :]
    B = np.atleast_2d(B)[None, :, :]
    A1x, A1y, A2x, A2y = A[..., 0], A[..., 1], A[..., 2], A[..., 3]
    B1x, B1y, B2x, B2y = B[..., 0], B[..., 1], B[..., 2], B[..., 3]
    apart = ((np.minimum(A1x, A2x) >= np.maximum(B1x, B2x)) | (np.maximum(A1x, A2x) <= np.minimum(B1x, B2x)) |
             (np.minimum(A1y, A2y) >= np.maximum(B1y, B2y)) | (np.maximum(A1y, A2y) <= np.minimum(B1y, B2y)))
    LB = np.sqrt((B2x - B1x) ** 2 + (B2y - B1y) ** 2)
    cA1 = (B2x - B1x) * (A1y - B1y) - (B2y - B1y) * (A1x - B1x)
    cA2 = (B2x - B1x) * (A2y - B1y) - (B2y - B1y) * (A2x - B1x)
    cB1 = (A2x - A1x) * (B1y - A1y) - (A2y - A1y) * (B1x - A1x)
    cB2 = (A2x - A1x) * (B2y - A1y) - (A2y - A1y) * (B2x - A1x)
    with np.errstate(divide="ignore", invalid="ignore"):
        dA1 = np.where(LB != 0, cA1 / np.where(LB != 0, LB, 1.0), np.nan)
        dA2 = np.where(LB != 0, cA2 / np.where(LB != 0, LB, 1.0), np.nan)
    flag = ~apart & (cA1 * cA2 < 0) & (cB1 * cB2 < 0)
    return flag, dA1, dA2


def GetInitRAndFiForInjection(SEO_R, SEO_Pr, InjectCL, Ek):
    """Injection point (azimuth, r, pr) on the closed orbit of energy Ek
    (src/FFAG_Distribution.py:1347-1414).  InjectCL a number: the azimuth in
    deg, r and pr by 4 x 4 Lagrange interpolation of the tables.  InjectCL an
    array (n, 2) of x, y points: the injection central line; the closed orbit
    of Ek (the tables' rows linearly interpolated in energy, My1p5DInterp)
    as a polyline over the azimuth axis, closed by repeating its second
    point; the first crossing of its segments with the line's (in segment
    order); the crossing point from the two ends' distances to the line's
    segment; pr of the orbit segment's start.  (The reference's last line
    indexes the scalar azimuth and raises for this branch; here the azimuth
    is returned as computed.)"""
    if isinstance(InjectCL, np.ndarray):
        Ek_axis, fi_axis = SEO_R[1:, 0], SEO_R[0, 1:]
        R, Pr = SEO_R[1:, 1:], SEO_Pr[1:, 1:]
        right = int(np.searchsorted(Ek_axis, Ek, side="right"))
        i0, i1 = right - 1, right
        if i0 < 0:
            i0, i1 = 0, 1
        if i1 > len(Ek_axis) - 1:
            i0, i1 = len(Ek_axis) - 2, len(Ek_axis) - 1
        x0, x1 = Ek_axis[i0], Ek_axis[i1]
        r_fi = (Ek - x1) / (x0 - x1) * R[i0] + (Ek - x0) / (x1 - x0) * R[i1]
        pr_fi = (Ek - x1) / (x0 - x1) * Pr[i0] + (Ek - x0) / (x1 - x0) * Pr[i1]
        traj = np.column_stack((r_fi * np.cos(fi_axis), r_fi * np.sin(fi_axis)))
        traj = np.vstack((traj, traj[1]))
        seo_seg, cl_seg = _segments(traj), _segments(InjectCL)
        flag, dA1, dA2 = _segment_crossings(seo_seg, cl_seg)
        ii, jj = np.nonzero(flag)
        if ii.size == 0:
            raise ValueError("the injection central line does not cross the closed orbit of this energy")
        i, j = ii[0], jj[0]
        pre_len, post_len = abs(dA1[i, j]), abs(dA2[i, j])
        total = pre_len + post_len
        P = ((pre_len - total) / (0 - total) * seo_seg[i, 0:2] + (pre_len - 0) / (total - 0) * seo_seg[i, 2:4])
        return float(np.arctan2(P[1], P[0])), float(np.hypot(P[0], P[1])), float(pr_fi[i])
    Ek_axis, fi_axis = SEO_R[1:, 0], SEO_R[0, 1:]
    theta = np.array([np.deg2rad(InjectCL)])
    r = Lagrange_interp_2D_vect(Ek_axis, fi_axis, SEO_R[1:, 1:], np.array([Ek]), theta)[0][0]
    pr = Lagrange_interp_2D_vect(Ek_axis, fi_axis, SEO_Pr[1:, 1:], np.array([Ek]), theta)[0][0]
    return theta[0], r, pr


# ------------------------------------------------------------ generators


def GenerateInitDistributionDtInjNew(SEOFileName, InjectionPosition, Ek_c, Emit, num_points, InjTimeNanoSec,
                                     LongitudeAlpha, LongitudeBeta, LongitudeT, acc_U0=100.0e3, acc_phi0=0.0,
                                     TwissParams=None, dist_types=("gauss", "gauss"), dx_xp_y_yp=(0.0, 0.0, 0.0, 0.0),
                                     Bunch_ID=0.0, bucket_obj=None, rng=None, device_out=None, seed=0):
    """One sub-bunch (src/FFAG_Distribution.py:1152-1345): returns (p-format
    matrix, distribution, centre (r, pr, z, pz, Ek, t), bucket_obj).
    device_out: a device float64 tensor of num_points x 16 rows; the rows are
    then drawn on the GPU (ffa_bunch_sample, Philox keyed by `seed` and the
    sub-bunch index Bunch_ID) and written there, and the returned matrix is
    that tensor."""
    from .seo import LoadSEOParams
    rng = rng if rng is not None else _default_rng
    eR, eZ, eFi = Emit[0] / 1000.0 / 1000.0, Emit[1] / 1000.0 / 1000.0, Emit[2]
    ini, bmap_path, _ = LoadSEOParams(os.path.join(SEOFileName, "SEO_ini.txt"), Ek_c)
    SEO_R = np.loadtxt(os.path.join(SEOFileName, "SEO_r.txt"), skiprows=1)
    SEO_Pr = np.loadtxt(os.path.join(SEOFileName, "SEO_pr.txt"), skiprows=1)
    Ek_c = ini[0]
    if isinstance(InjectionPosition, dict):
        fi_c, r_c, pr_c = InjectionPosition["fi"], InjectionPosition["r"], InjectionPosition["pr"]
    elif isinstance(InjectionPosition, str):           # a central-line file: x, y after one header line
        fi_c, r_c, pr_c = GetInitRAndFiForInjection(SEO_R, SEO_Pr, np.loadtxt(InjectionPosition, skiprows=1), Ek_c)
    elif isinstance(InjectionPosition, (float, int)):
        fi_c, r_c, pr_c = GetInitRAndFiForInjection(SEO_R, SEO_Pr, float(InjectionPosition), Ek_c)
    else:
        raise ValueError("Unsupported type for InjectionPosition")
    if TwissParams is not None:
        bZ, bR, aZ, aR = TwissParams
    else:
        bZ, bR, aZ, aR = LoadSEOBetaFunc(SEOFileName, Ek_c, fi_c)
    ttype, ltype = dist_types
    if ltype == "match" and bucket_obj is None:
        from .bucket import FFAG_bucket
        bucket_obj = FFAG_bucket(bmap_path, Ek0=Ek_c, fi0=acc_phi0, U0=acc_U0, step_t=20e-9, step_N=18000)
    if ltype == "kv":
        eFi *= 2
    tw_fi = TwissContainer(LongitudeAlpha, LongitudeBeta, eFi)
    dist = CustomDist3D(create_distribution(ttype, twiss_transverse=(TwissContainer(aR, bR, eR),
                                                                       TwissContainer(aZ, bZ, eZ))),
                        create_distribution(ltype, twiss_longitudinal=tw_fi))
    rc, prc, zc, pzc = r_c + dx_xp_y_yp[0], pr_c + dx_xp_y_yp[1], dx_xp_y_yp[2], dx_xp_y_yp[3]
    if device_out is not None and ltype == "match":
        # the bucket's rejection sampling runs on the host; the rows go to the device
        import torch
        a, dist, centre, bucket_obj = GenerateInitDistributionDtInjNew(
            SEOFileName, InjectionPosition, Ek_c, Emit, num_points, InjTimeNanoSec, LongitudeAlpha, LongitudeBeta,
            LongitudeT, acc_U0, acc_phi0, TwissParams, dist_types, dx_xp_y_yp, Bunch_ID, bucket_obj, rng)
        device_out.copy_(torch.from_numpy(a))
        return device_out, dist, centre, bucket_obj
    if device_out is not None:
        _sample_on_device(device_out, num_points, ttype, ltype, ((aR, bR, eR), (aZ, bZ, eZ),
                          (LongitudeAlpha, LongitudeBeta, eFi)), LongitudeT,
                          math.sqrt(eFi / LongitudeBeta), (rc, prc, zc, pzc, Ek_c, InjTimeNanoSec), fi_c,
                          Bunch_ID, seed)
        return device_out, dist, (rc, prc, zc, pzc, Ek_c, InjTimeNanoSec), bucket_obj
    r, pr, z, pz, t_inj, Ek = dist.sample(num_points, rng)
    if ltype == "UniformGauss":
        sigma = math.sqrt(eFi / LongitudeBeta)
        t_inj = rng.uniform(-0.5 * LongitudeT, 0.5 * LongitudeT, num_points)
        Ek = rng.normal(0.0, sigma, num_points)
    elif ltype == "match":       # src/FFAG_Distribution.py:1270-1275
        t_inj, Ek_MeV, _ = bucket_obj.scatter_filter_by_span(num_points, LongitudeT, rng=rng)
        Ek = Ek_MeV - Ek_c
    a = np.zeros((num_points, 16))
    a[:, COLUMNS["r"]] = r + rc
    a[:, COLUMNS["vr"]] = pr + prc
    a[:, COLUMNS["z"]] = z + zc
    a[:, COLUMNS["vz"]] = pz + pzc
    a[:, COLUMNS["fi"]] = fi_c
    a[:, 5] = Ek + Ek_c
    a[:, COLUMNS["inj_t"]] = t_inj + InjTimeNanoSec
    a[:, 13] = Bunch_ID
    a[:, 14] = np.arange(num_points)
    a[:, 15] = np.arange(num_points)
    return a, dist, (rc, prc, zc, pzc, Ek_c, InjTimeNanoSec), bucket_obj


def _sample_on_device(out, n, ttype, ltype, twiss, length, sigma, centre, fi, bunch_id, seed, id0=0):
    """One ffa_bunch_sample call writing n p-format rows into `out` (device
    float64, n x 16, contiguous)."""
    import ctypes
    import torch
    from . import _lib
    if out.dtype != torch.float64 or not out.is_cuda or not out.is_contiguous() or tuple(out.shape) != (n, 16):
        raise ValueError("device_out must be a contiguous CUDA float64 tensor of shape (num_points, 16)")
    for t, kind in ((ttype, "transverse"), (ltype, "longitudinal")):
        if t not in _lib.DIST_TYPES or (kind == "transverse" and t == "UniformGauss"):
            raise ValueError(f"{kind} distribution {t!r} is not built on the device")
    d = _lib.BunchDesc()
    d.n, d.id0, d.seed, d.sub_bunch = int(n), int(id0), int(seed) & ((1 << 64) - 1), int(bunch_id)
    d.transverse, d.longitudinal = _lib.DIST_TYPES[ttype], _lib.DIST_TYPES[ltype]
    d.cut_off = -1.0
    for p in range(3):
        for k in range(3):
            d.twiss[p][k] = float(twiss[p][k])
    d.uniform_length, d.uniform_sigma = float(length), float(sigma)
    for k in range(6):
        d.centre[k] = float(centre[k])
    d.fi, d.bunch_id, d.out = float(fi), float(bunch_id), out.data_ptr()
    with torch.cuda.device(out.device):
        _lib.check(_lib.lib().ffa_bunch_sample(ctypes.byref(d), None,
                                                torch.cuda.current_stream(out.device).cuda_stream),
                   "ffa_bunch_sample")


def _emap_paint_params(path):
    with open(path) as f:
        content = f.read()
    get = lambda key: (float(m.group(1)) if (m := re.search(key + r" = ([\d.eE+-]+)", content)) else None)
    return get("gap_azimuth"), get("acc_phi_paint"), get("acc_voltage_paint")


def GenerateBunches(BunchPara, rng=None, device=None):
    """All painted sub-bunches, stacked (src/FFAG_Distribution.py:1542-1640).
    BunchPara holds the reference's keys (SEO, InjectEk, InjPosition,
    ParticleNum, TransverseREmit, TransverseZEmit, LongitudeT, LongitudeDEk,
    InjTimeNanoSec, TransverseDistType, LongitudeDistType, PaintEnable,
    PaintMaxNum, PaintTimeInterval, PaintCurve, EmapPATHName) and optionally
    Seed.  device: draw the particles on that GPU (ffa_bunch_sample) and
    return a device float64 tensor; the host side (SEO tables, painting
    offsets) is the same."""
    if device is not None:
        import torch
        num = int(BunchPara["ParticleNum"])
        curve_n = 1
        if BunchPara["PaintEnable"]:
            c_ = np.loadtxt(BunchPara["PaintCurve"], skiprows=1)
            curve_n = int(min(np.floor(np.max(c_[:, 0]) / BunchPara["PaintTimeInterval"]), BunchPara["PaintMaxNum"]))
        out_dev = torch.empty((curve_n * num, 16), dtype=torch.float64, device=device)
    if rng is None:
        rng = np.random.default_rng(BunchPara.get("Seed"))
    _, acc_phi0, acc_V0 = _emap_paint_params(BunchPara["EmapPATHName"])
    if BunchPara["PaintEnable"]:
        curve = np.loadtxt(BunchPara["PaintCurve"], skiprows=1)
        nb = int(min(np.floor(np.max(curve[:, 0]) / BunchPara["PaintTimeInterval"]), BunchPara["PaintMaxNum"]))
    else:
        curve, nb = None, 1
    LT, LdE = BunchPara["LongitudeT"], BunchPara["LongitudeDEk"]
    out = []
    bucket = None
    for i in range(nb):
        t_inj = i * BunchPara["PaintTimeInterval"]
        if curve is not None:
            off = tuple(np.interp(t_inj, curve[:, 0], curve[:, c]) for c in (1, 2, 3, 4))
        else:
            off = (0, 0, 0, 0)
        sub, _, _, bucket = GenerateInitDistributionDtInjNew(
            BunchPara["SEO"], BunchPara["InjPosition"], BunchPara["InjectEk"],
            [BunchPara["TransverseREmit"], BunchPara["TransverseZEmit"], LT * LdE / 16], BunchPara["ParticleNum"],
            t_inj, 0.0, LT / LdE, LT, acc_U0=acc_V0, acc_phi0=acc_phi0,
            dist_types=(BunchPara["TransverseDistType"], BunchPara["LongitudeDistType"]), dx_xp_y_yp=off,
            Bunch_ID=i, bucket_obj=bucket, rng=rng,
            device_out=None if device is None else out_dev[i * num:(i + 1) * num],
            seed=int(BunchPara.get("Seed") or 0))
        out.append(sub)
    return out_dev if device is not None else np.vstack(out)
