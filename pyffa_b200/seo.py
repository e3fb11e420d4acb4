"""Closed-orbit (SEO) search, tunes and the SEO text files, batched on the GPU.

Drop-in for the reference's FFAG_SearchSEO (src/FFAG_track.py:1142-1621) as
driven by examples/main_SEO.py, and for LoadSEOParams
(src/FFAG_Distribution.py:1417-1427), which the tracking driver and the
space-charge step read back.

The reference integrates one trajectory at a time in Python (RK4 in the
azimuth, h = 0.001 rad, FunctionForSEO) and iterates per energy.  Here every
azimuth track of one iteration — all energies, and the perturbed companions
of the Newton step and of the tune estimate — is one launch of
ffa_theta_track, one GPU thread per trajectory; the host runs the same
iteration rules as the reference, per energy, in lockstep:

1. start radius from the sector-mean field by 100 bisection steps
   (SearchSEOUsingInitialEkVect / func_get_R_B0);
2. fixed-point averaging of start and end of a one-sector track until both
   r and pr close to 1e-5 (up to 200 passes per starting pr0, trying
   pr0 = 0, +-0.02, ... +-0.14 after a NaN);
3. Newton refinement with finite-difference Jacobian (TrackBunchSEO), up to 25
   passes, |dr/r| < 1e-8;
4. a full-turn track for r(th), pr(th) and their values at 90/180/270 degrees;
5. tunes from the one-sector transfer-matrix traces (GetQrQz) and the
   revolution frequency and perimeter from the arc length (GetFreq).

SEO_ini.txt keeps the reference's columns, rounding (3 decimals for the
tunes, frequency and mean radius, 8 for the rest) and padding; SEO_r.txt and
SEO_pr.txt keep its matrix layout (first row: first energy, then the azimuth
points; one row per energy).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .constants import FFAG_ConversionTools

PR0_LIST = [0.00, 0.02, -0.02, 0.04, -0.04, 0.06, -0.06, 0.08, -0.08, 0.10, -0.10, 0.12, -0.12, 0.14, -0.14]
TITLES = ["Ek_index", "Ek_value(MeV)", "Qr", "Qz", "OrbitFreq(Hz)", "MeanR(m)",
          "r0(m)", "pr0", "Perimeter(m)", "r360(m)", "pr360",
          "r90(m)", "pr90", "r180(m)", "pr180", "r270(m)", "pr270"]


class ThetaTracker:
    """Batched azimuth-domain tracks through the analytic field (ffa_theta_track)."""

    def __init__(self, bmap, q, device=None):
        import torch
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.fm = bmap.device_map(self.dev)
        self.q = float(q)

    def run(self, x0, t_end, h, time_mode=0, traj=False, traj_cols=2):
        """x0: (m, 5) r, pr, z, pz, P.  Returns (x1 (m, 4), traj (m, n,
        traj_cols) or None, t_points) for the reference's n = int(t_end / h)
        azimuth points; 7 columns add z, pz and the field Bz, Br, Bfi."""
        import torch
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, 5)
        m = x0.shape[0]
        n = int((t_end - 0) / h)
        t_points = np.linspace(0, t_end, n)
        f64 = dict(dtype=torch.float64, device=self.dev)
        tx0 = torch.from_numpy(x0).to(self.dev)
        tx1 = torch.empty((m, 4), **f64)
        ttr = torch.empty((m, n, traj_cols), **f64) if traj else None
        d = _lib.ThetaTrackDesc()
        d.m, d.n_points, d.time_mode, d.t_end, d.q = m, n, int(time_mode), float(t_end), self.q
        d.traj_cols = traj_cols
        d.x0, d.x1 = tx0.data_ptr(), tx1.data_ptr()
        d.traj = ttr.data_ptr() if traj else None
        stream = torch.cuda.current_stream(self.dev)
        _lib.check(_lib.lib().ffa_theta_track(self.fm.handle, ctypes.byref(d), stream.cuda_stream),
                   "ffa_theta_track")
        x1 = tx1.cpu().numpy()
        return x1, (ttr.cpu().numpy() if traj else None), t_points


def _interp_extrap(x, y, xi):
    from scipy.interpolate import interp1d
    return interp1d(x, y, kind="linear", fill_value="extrapolate")(xi)


class FFAG_SearchSEO:
    def __init__(self, GlobalParas, device=None, tracker=None):
        """`tracker` (default: the GPU ThetaTracker) is anything with the
        ThetaTracker.run interface."""
        self.GlobalParas = GlobalParas
        self.bm = GlobalParas.Bmap
        self.q = GlobalParas.q
        self.N = self.bm.Nsectors
        self.tracker = tracker if tracker is not None else ThetaTracker(self.bm, self.q, device)
        self.conv = FFAG_ConversionTools()
        if getattr(getattr(GlobalParas, "BHarmonics", None), "enable_flag", False):
            raise NotImplementedError("field-error harmonics are not supported by the GPU closed-orbit search")

    # ------------------------------------------------------------ pieces
    def initial_radius(self, Ek):
        """Bisection of r - P / q / <B>(r) over [r_min, r_max], 100 passes
        (FFAG_Algorithm.BiSection with func_get_R_B0, src/FFAG_MathTools.py:479-489,
        src/FFAG_track.py:1804-1810), for each energy."""
        f1 = self.bm.f1
        if f1 is None:
            raise ValueError("the lattice JSON has no Bmap.Bmean: run FFAG_Bfield_analytical.UpdataConfig first")
        out = []
        for E in np.atleast_1d(Ek):
            P = self.conv.Ek2P(E)
            func = lambda r: r - P / self.q / f1(r)
            xl, xr = self.bm.r_min, self.bm.r_max
            xm = float("nan")
            for _ in range(100):
                xm = (xl + xr) / 2
                yl, ym = func(xl), func(xm)
                if ym * yl < 0:
                    xr = xm
                else:
                    xl = xm
            out.append(xm)
        return np.array(out, dtype=np.float64)

    def _sector(self):
        return np.pi * 2 / self.N

    def fixed_point(self, Ek, r0_an, h=0.001, delta_r0_ini=0.0):
        """Step 2 for all energies in lockstep; returns (r0, pr0)."""
        Ek = np.asarray(Ek, dtype=np.float64)
        m = len(Ek)
        P = np.array([self.conv.Ek2P(E) for E in Ek])
        pri = np.zeros(m, dtype=np.int64)          # index into PR0_LIST
        k = np.zeros(m, dtype=np.int64)
        r0 = r0_an + delta_r0_ini
        pr0 = np.full(m, PR0_LIST[0])
        state = np.zeros(m, dtype=np.int64)         # 0 running, 1 found, 2 failed
        while (state == 0).any():
            act = np.nonzero(state == 0)[0]
            x0 = np.stack([r0[act], pr0[act], np.zeros(len(act)), np.zeros(len(act)), P[act]], axis=1)
            x1, _, _ = self.tracker.run(x0, self._sector(), h)
            for j, e in enumerate(act):
                rs, ps = x0[j, 0], x0[j, 1]
                re, pe = x1[j, 0], x1[j, 1]
                r0[e], pr0[e] = (rs + re) / 2, (ps + pe) / 2
                k[e] += 1
                if np.isnan(re) or np.isnan(pe):
                    pri[e] += 1
                    k[e] = 0
                    if pri[e] >= len(PR0_LIST):
                        state[e] = 2
                    else:
                        r0[e] = r0_an[e] + delta_r0_ini
                        pr0[e] = PR0_LIST[pri[e]]
                    continue
                if abs(rs - re) < 1e-5 and abs(ps - pe) < 1e-5:
                    state[e] = 1
                    continue
                if k[e] >= 200:
                    pri[e] += 1
                    k[e] = 0
                    if pri[e] >= len(PR0_LIST):
                        state[e] = 2
                    else:
                        r0[e] = r0_an[e] + delta_r0_ini
                        pr0[e] = PR0_LIST[pri[e]]
        if (state == 2).any():
            bad = Ek[state == 2]
            raise RuntimeError(f"No close orbit solution found for {bad.tolist()} MeV.")
        return r0, pr0

    def newton(self, Ek, r0, p0, h=0.001):
        """Step 3 (TrackBunchSEO, src/FFAG_track.py:1169-1202) in lockstep."""
        Ek = np.asarray(Ek, dtype=np.float64)
        m = len(Ek)
        P = np.array([self.conv.Ek2P(E) for E in Ek])
        r0, p0 = r0.copy(), p0.copy()
        dr, dp = r0 * 0.0001, 0.001
        active = np.ones(m, dtype=bool)
        for _ in range(25):
            act = np.nonzero(active)[0]
            if len(act) == 0:
                break
            x0 = np.zeros((3 * len(act), 5))
            for j, e in enumerate(act):
                x0[3 * j] = [r0[e], p0[e], 0, 0, P[e]]
                x0[3 * j + 1] = [r0[e] + dr[e], p0[e], 0, 0, P[e]]
                x0[3 * j + 2] = [r0[e], p0[e] + dp, 0, 0, P[e]]
            x1, _, _ = self.tracker.run(x0, self._sector(), h, time_mode=1)
            for j, e in enumerate(act):
                r0f, p0f = x1[3 * j, 0], x1[3 * j, 1]
                r1f, p1f = x1[3 * j + 1, 0], x1[3 * j + 1, 1]
                r2f, p2f = x1[3 * j + 2, 0], x1[3 * j + 2, 1]
                a11 = (r1f - r0f) / dr[e]
                a12 = (r2f - r0f) / dp
                a21 = (p1f - p0f) / dr[e]
                a22 = (p2f - p0f) / dp
                a11p, a22p = a11 - 1, a22 - 1
                det = a11p * a22p - a12 * a21
                if np.abs((r0f - r0[e]) / r0[e]) < 1e-8:
                    active[e] = False
                    continue
                re = r0[e] + a22p / det * (r0[e] - r0f) - a12 / det * (p0[e] - p0f)
                pe = p0[e] + a11p / det * (p0[e] - p0f) - a21 / det * (r0[e] - r0f)
                r0[e], p0[e] = re, pe
        return r0, p0

    def tunes(self, Ek, r0, pr0, h=0.001):
        """GetQrQz (src/FFAG_track.py:1257-1309) for every energy: (Qr, Qz,
        frequency, mean radius, perimeter)."""
        Ek = np.asarray(Ek, dtype=np.float64)
        m = len(Ek)
        P = np.array([self.conv.Ek2P(E) for E in Ek])
        drr, dpp, dzz, dpz = 1e-6, 1e-6, 1e-7, 1e-7
        x0 = np.zeros((5 * m, 5))
        for e in range(m):
            x0[5 * e] = [r0[e], pr0[e], 0.0, 0.0, P[e]]
            x0[5 * e + 1] = [r0[e] + drr, pr0[e], 0.0, 0.0, P[e]]
            x0[5 * e + 2] = [r0[e], pr0[e] + dpp, 0.0, 0.0, P[e]]
            x0[5 * e + 3] = [r0[e], pr0[e], 0.0 + dzz, 0.0, P[e]]
            x0[5 * e + 4] = [r0[e], pr0[e], 0.0, 0.0 + dpz, P[e]]
        x1, tr, t_points = self.tracker.run(x0, self._sector(), h, traj=True)
        out = np.zeros((m, 5))
        for e in range(m):
            r1, p1, z1, pz1 = x1[5 * e, 0], x1[5 * e, 1], 0.0, 0.0
            freq, perim = self.GetFreq(t_points, tr[5 * e, :, 0], tr[5 * e, :, 1], Ek[e])
            mean_r = np.mean(tr[5 * e, :, 0])
            r2 = x1[5 * e + 1, 0]
            p3 = x1[5 * e + 2, 1]
            z2 = x1[5 * e + 3, 2]
            pz3 = x1[5 * e + 4, 3]
            a11 = (r2 - r1) / drr
            a22 = (p3 - p1) / dpp
            b11 = (z2 - z1) / dzz
            b22 = (pz3 - pz1) / dpz
            Qr = np.arccos((a11 + a22) / 2) / (2 * np.pi) * self.N
            Qz = np.arccos((b11 + b22) / 2) / (2 * np.pi) * self.N
            out[e] = [Qr, Qz, freq, mean_r, perim]
        return out

    def GetFreq(self, fi_SEO, r_SEO, pr_SEO, Ek_value):
        """Revolution frequency and perimeter from one sector's arc length
        (src/FFAG_track.py:1359-1378; the perimeter sums in sequence)."""
        rp = pr_SEO / (np.sqrt(1 - pr_SEO ** 2)) * r_SEO
        arc = np.sqrt(r_SEO ** 2 + rp ** 2) * (fi_SEO[2] - fi_SEO[1])
        perim = 0
        for v in arc[:-1]:
            perim = perim + v
        perim = perim * self.N
        v = self.conv.Ek2v(Ek_value)
        return 1 / (perim / v), perim

    # ------------------------------------------------------------ driver
    def search(self, EkRange, h=0.001):
        """Every per-energy quantity of the SEO files."""
        Ek = np.asarray(EkRange, dtype=np.float64)
        r_an = self.initial_radius(Ek)
        r0, pr0 = self.fixed_point(Ek, r_an, h)
        r0, pr0 = self.newton(Ek, r0, pr0, h)
        P = np.array([self.conv.Ek2P(E) for E in Ek])
        x0 = np.stack([r0, pr0, np.zeros_like(r0), np.zeros_like(r0), P], axis=1)
        x1, tr, t_full = self.tracker.run(x0, np.pi * 2, 0.001, traj=True)
        q = self.tunes(Ek, r0, pr0, h)
        rows = np.zeros((len(Ek), 17))
        for e in range(len(Ek)):
            r_of, pr_of = tr[e, :, 0], tr[e, :, 1]
            at = [_interp_extrap(t_full, y, np.deg2rad(a)) for a in (90.0, 180.0, 270.0) for y in (r_of, pr_of)]
            rows[e] = [e, Ek[e], q[e, 0], q[e, 1], q[e, 2], q[e, 3], r0[e], pr0[e], q[e, 4],
                       r_of[-1], pr_of[-1], *at]
        return {"table": rows, "fi": t_full, "r": tr[:, :, 0], "pr": tr[:, :, 1], "r0_analytical": r_an}

    def SearchSEOsControllerVect(self, EkRange, SavedataFlag=True, h=0.001):
        """Searches every energy and writes SEO_ini.txt, SEO_r.txt and
        SEO_pr.txt into <Bmap folder>/<GlobalParas.SEO_SaveFold>; returns
        that folder (src/FFAG_track.py:1380-1512)."""
        res = self.search(EkRange, h)
        if not SavedataFlag:
            return None
        fold = os.path.join(self.bm.BmapFoldName, self.GlobalParas.SEO_SaveFold)
        os.makedirs(fold, exist_ok=True)
        write_seo_files(fold, self.bm.BmapFoldName, h, res["table"], res["fi"], np.asarray(EkRange, np.float64),
                        res["r"], res["pr"])
        return fold


def format_seo_ini(table, bmap_folder, h):
    """SEO_ini.txt text (src/FFAG_track.py:1455-1488)."""
    t = np.asarray(table, dtype=float).copy()
    t[:, 2:6] = np.round(t[:, 2:6], 3)
    t[:, 6:] = np.round(t[:, 6:], 8)
    rows = [TITLES] + t.tolist()
    widths = [max(len(str(row[i])) for row in rows) for i in range(len(rows[0]))]
    lines = ["  ".join([str(v).ljust(w) for v, w in zip(row, widths)]) for row in rows]
    lines.insert(0, "Bmap foldname=" + bmap_folder + ", step h = %.6f rad" % (h,))
    return "\n".join(lines)


def write_seo_files(fold, bmap_folder, h, table, fi, Ek, r, pr):
    with open(os.path.join(fold, "SEO_ini.txt"), "w") as f:
        f.write(format_seo_ini(table, bmap_folder, h))
    head = np.hstack((Ek[0], fi))
    for name, unit, data in (("SEO_r.txt", "unitR=m", r), ("SEO_pr.txt", "unitPr=1", pr)):
        mat = np.vstack((head, np.hstack((Ek[:, None], data))))
        with open(os.path.join(fold, name), "w") as f:
            f.write(f"unitEk=MeV, unitFi=deg, {unit}\n")
        with open(os.path.join(fold, name), "a") as f:
            np.savetxt(f, mat)


def LoadSEOParams(SEOFileName, Ek_c):
    """([Ek, r0, pr0, T_rev], Bmap folder, SEO table) at energy Ek_c from
    SEO_ini.txt (src/FFAG_Distribution.py:1417-1427; linear interpolation
    between the two bracketing energies, end intervals extended)."""
    path = os.path.dirname(os.path.dirname(SEOFileName))
    data = np.loadtxt(SEOFileName, skiprows=2)
    data = np.atleast_2d(data)
    Ek0, r0, pr0, T0 = data[:, 1], data[:, 6], data[:, 7], 1 / data[:, 4]

    def lin(X, Y, xi):
        right = int(np.searchsorted(X, xi, side="right"))
        left = right - 1
        if left < 0:
            i0, i1 = 0, 1
        elif right > len(X) - 1:
            i0, i1 = len(X) - 2, len(X) - 1
        else:
            i0, i1 = left, right
        return Y[i0] + (xi - X[i0]) / (X[i1] - X[i0]) * (Y[i1] - Y[i0])

    return np.array([Ek_c, lin(Ek0, r0, Ek_c), lin(Ek0, pr0, Ek_c), lin(Ek0, T0, Ek_c)]), path, data


def main_SEO(json_path: str, device=None) -> str:
    """examples/main_SEO.py: energies start_Ek..end_Ek by delta_Ek plus
    extra_Ek, the map folder's config_Bmap.json (with Bmap.Bmean), the SEO
    files and the Twiss tables into <map folder>/<SEO_folder>, and the
    configuration copied there as config_SEO.json.  Returns the SEO folder."""
    import json

    from .fields import FFAG_Bfield_analytical
    from .constants import FFAG_GlobalParameters
    with open(json_path) as f:
        cfg = json.load(f)
    c = cfg["config"]
    Ek = np.arange(c["start_Ek"], c["end_Ek"] + c["delta_Ek"], c["delta_Ek"])
    Ek = np.sort(np.concatenate((Ek, np.array(c.get("extra_Ek", []), dtype=np.float64))))
    harm = cfg.get("BHarmonics", {"enable": False, "harmonics": []})
    if harm.get("enable"):
        raise NotImplementedError("field-error harmonics are not supported by the GPU closed-orbit search")
    gp = FFAG_GlobalParameters()
    gp.AddBMap(FFAG_Bfield_analytical(os.path.join(c["Bmap_path"], "config_Bmap.json"), 0, AddNumricalMap=False))
    gp.SEO_SaveFold = c["SEO_folder"]
    finder = FFAG_SearchSEO(gp, device)
    fold = finder.SearchSEOsControllerVect(Ek)
    CalcBetaFunc(fold, Ek, gp, tracker=finder.tracker)
    with open(os.path.join(fold, "config_SEO.json"), "w") as f:
        json.dump(cfg, f, indent=2, sort_keys=True)
    return fold


# ------------------------------------------------------------------ Twiss


def _two_points(X, xi):
    """find_two_points_non_uniform_vect (src/FFAG_MathTools.py:59-82): bracketing
    indices, end intervals extended."""
    xi = np.atleast_1d(xi)
    right = np.searchsorted(X, xi, side="right")
    left = right - 1
    i0, i1 = left.copy(), right.copy()
    lo = left < 0
    i0[lo], i1[lo] = 0, 1
    hi = right > len(X) - 1
    i0[hi], i1[hi] = len(X) - 2, len(X) - 1
    return i0, i1


def _interp_2p5d(M, ax0, ax1, fi0, pid):
    """My2p5DInterp (src/FFAG_MathTools.py:329-364): bilinear in (azimuth
    step, particle id) of M[step, id, :], the reference's weight formulas."""
    a0, a1 = _two_points(ax0, fi0)
    b0, b1 = _two_points(ax1, pid)
    x0, x1, y0, y1 = ax0[a0], ax0[a1], ax1[b0], ax1[b1]
    L00 = (fi0 - x1) * (pid - y1) / (x0 - x1) / (y0 - y1)
    L01 = (fi0 - x1) * (pid - y0) / (x0 - x1) / (y1 - y0)
    L10 = (fi0 - x0) * (pid - y1) / (x1 - x0) / (y0 - y1)
    L11 = (fi0 - x0) * (pid - y0) / (x1 - x0) / (y1 - y0)
    return (L00[:, None] * M[a0, b0, :] + L01[:, None] * M[a0, b1, :] + L10[:, None] * M[a1, b0, :]
            + L11[:, None] * M[a1, b1, :])


def _find_coef(r1_s, pr1_s, r1_e, pr1_e, r2_s, pr2_s, r2_e, pr2_e):
    """Transfer-matrix elements from two trajectories by Cramer's rule
    (FFAG_BetaFuncCalc.find_coef, src/FFAG_BetaFunc.py:26-43)."""
    m00 = np.array([[r1_s, pr1_s, 0, 0], [0, 0, r1_s, pr1_s], [r2_s, pr2_s, 0, 0], [0, 0, r2_s, pr2_s]])
    rhs = np.array([r1_e, pr1_e, r2_e, pr2_e])
    d0 = np.linalg.det(m00)
    out = []
    for col in range(4):
        m = m00.copy()
        m[:, col] = rhs
        out.append(np.linalg.det(m) / d0)
    return tuple(out)


def load_seo_params_vect(SEOFileName, Ek_arr):
    """FFAG_BetaFuncCalc.LoadSEOParams (src/FFAG_BetaFunc.py:17-24)."""
    path = os.path.dirname(os.path.dirname(SEOFileName))
    data = np.atleast_2d(np.loadtxt(SEOFileName, skiprows=2))
    Ek0, r0, pr0 = data[:, 1], data[:, 6], data[:, 7]
    Ek_arr = np.atleast_1d(np.asarray(Ek_arr, dtype=np.float64))
    i0, i1 = _two_points(Ek0, Ek_arr)
    lin = lambda Y: Y[i0] + (Ek_arr - Ek0[i0]) / (Ek0[i1] - Ek0[i0]) * (Y[i1] - Y[i0])
    return np.column_stack([Ek_arr, lin(r0), lin(pr0)]), path, data


def CalcBetaFunc(SEOPATHName, Ek_arr, GlobalParas=None, tracker=None, device=None, write=True):
    """Twiss functions along one sector for every energy
    (FFAG_BetaFuncCalc.CalcBetaFunc, src/FFAG_BetaFunc.py:45-240): five
    trajectories per energy (the closed orbit and r, pr, z, pz nudged by
    1e-7) tracked over two sectors in one batched launch; at 1000 azimuths
    the one-sector transfer matrices from the interpolated trajectories give
    beta = m12 / sin(mu), alpha = (m11 - m22) / (2 sin(mu)).  Writes
    BetaFuncR/Z.txt, AlphaFuncR/Z.txt and the field along the orbit Bz/Br/Bf.txt
    into SEOPATHName; returns (beta_r, beta_z, alpha_r, alpha_z, fi_deg)."""
    from .constants import FFAG_GlobalParameters
    from .fields import FFAG_Bfield_analytical
    h = 0.001
    Ek_arr = np.asarray(Ek_arr, dtype=np.float64)
    nE = len(Ek_arr)
    ini, bmap_path, _ = load_seo_params_vect(os.path.join(SEOPATHName, "SEO_ini.txt"), Ek_arr)
    conv = FFAG_ConversionTools()
    if GlobalParas is None:
        GlobalParas = FFAG_GlobalParameters()
        GlobalParas.AddBMap(FFAG_Bfield_analytical(os.path.join(bmap_path, "config_Bmap.json"), 0,
                                                   AddNumricalMap=False))
    bm = GlobalParas.Bmap
    if tracker is None:
        tracker = ThetaTracker(bm, GlobalParas.q, device)
    P0 = conv.Ek2P(ini[:, 0])
    base = np.column_stack((ini[:, 1], ini[:, 2], np.zeros(nE), np.zeros(nE), P0))
    delta = np.array([[0, 0, 0, 0, 0], [1e-7, 0, 0, 0, 0], [0, 1e-7, 0, 0, 0], [0, 0, 1e-7, 0, 0],
                      [0, 0, 0, 1e-7, 0]], dtype=np.float64)
    x0 = np.repeat(base, 5, axis=0) + np.tile(delta, (nE, 1))
    sector = np.pi * 2 / bm.Nsectors
    t_end = np.pi * 2 * 2 / bm.Nsectors + 0
    _, tr, tp = tracker.run(x0, t_end, h, time_mode=1, traj=True, traj_cols=7)
    hs = tp[1] - tp[0]
    times = np.zeros(tr.shape[1])
    for i in range(1, len(times)):
        times[i] = times[i - 1] + hs
    M = np.concatenate((times[None, :, None].repeat(x0.shape[0], axis=0).transpose(1, 0, 2),
                        tr[:, :, 0:4].transpose(1, 0, 2)), axis=2)       # [step, id, (t, r, pr, z, pz)]
    ids = np.arange(x0.shape[0], dtype=np.float64)
    fi0 = np.linspace(0, sector, 1000)
    br, bz, ar, az = (np.zeros((nE, 1000)) for _ in range(4))
    for n in range(1000):
        ts = fi0[n]
        te = ts + sector
        s = _interp_2p5d(M, times, ids, np.full(len(ids), ts), ids)
        e = _interp_2p5d(M, times, ids, np.full(len(ids), te), ids)
        for k in range(nE):
            xs = s[k * 5 + 1:(k + 1) * 5, 1:5] - s[k * 5, 1:5]
            xe = e[k * 5 + 1:(k + 1) * 5, 1:5] - e[k * 5, 1:5]
            a11, a12, a21, a22 = _find_coef(xs[0, 0], xs[0, 1], xe[0, 0], xe[0, 1],
                                            xs[1, 0], xs[1, 1], xe[1, 0], xe[1, 1])
            b11, b12, b21, b22 = _find_coef(xs[2, 2], xs[2, 3], xe[2, 2], xe[2, 3],
                                            xs[3, 2], xs[3, 3], xe[3, 2], xe[3, 3])
            cr, cz = (a11 + a22) / 2, (b11 + b22) / 2
            sr, sz = np.sqrt(1 - cr ** 2), np.sqrt(1 - cz ** 2)
            if a12 * sr < 0:
                sr = sr * (-1)
            if b12 * sz < 0:
                sz = sz * (-1)
            br[k, n], bz[k, n] = a12 / sr, b12 / sz
            ar[k, n], az[k, n] = (a11 - a22) / sr / 2, (b11 - b22) / sz / 2
    fi_deg = np.rad2deg(fi0)
    if write:
        a = np.insert(Ek_arr, 0, 0)
        files = [("BetaFuncR.txt", "unitBeta=m", np.vstack((fi_deg, br))),
                 ("BetaFuncZ.txt", "unitBeta=m", np.vstack((fi_deg, bz))),
                 ("AlphaFuncR.txt", "unitAlpha=1", np.vstack((fi_deg, ar))),
                 ("AlphaFuncZ.txt", "unitAlpha=m", np.vstack((fi_deg, az))),
                 ("Bz.txt", "unitB=T", np.vstack((times[None, :], tr[::5, :, 4]))),
                 ("Br.txt", "unitB=T", np.vstack((times[None, :], tr[3::5, :, 5]))),
                 ("Bf.txt", "unitB=T", np.vstack((times[None, :], tr[3::5, :, 6])))]
        for name, unit, mat in files:
            with open(os.path.join(SEOPATHName, name), "w") as f:
                f.write(f"unitEk=MeV, unitFi=deg, {unit}\n")
            with open(os.path.join(SEOPATHName, name), "a") as f:
                np.savetxt(f, np.column_stack((a, mat)))
    return br, bz, ar, az, fi_deg
