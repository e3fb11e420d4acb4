"""RF-bucket-matched longitudinal distribution (FFAG_bucket,
src/FFAG_bucket.py:1-457), the 'match' longitudinal type of the bunch
generator (src/FFAG_Distribution.py:1270-1275).

The longitudinal motion about the synchronous particle at energy Ek0 with
RF phase fi0 and voltage U0 is the Hamiltonian flow

    dzd/dt  = -(Tc - T(Ek0 + dEk)) / Tc
    ddEk/dt = U0 (sin(fi0 + w0 zd) - sin(fi0)) / Tc / 1e6       [MeV/s]

(zd the time offset, T(Ek) the revolution period from the closed-orbit
table, Tc = T(Ek0), w0 = 2 pi f(Ek0); DynamicFunc2_njit, :27-44).  The class
integrates 20 starting points on a ring round the unstable fixed point and
20 on the centre line, forward and backward in time (RK4, step step_t,
step_N steps), marks each trajectory stable or not (it never reaches
|w0 zd| = pi and its amplitudes do not grow by more than 20 % between the
halves of the run), takes the sampling box from the stable trajectories,
builds H(q, p) = -∫B dq + ∫A dp on a grid (trapezoids), relates each
centre-line trajectory's energy H to its time span, and draws particles
uniformly in the box with H >= H(target span) (scatter_filter_by_span).

The reference draws with an unseeded numpy Generator; here the draws take
a caller's Generator (seeded by the bunch generator)."""
from __future__ import annotations

import os

import numpy as np


def _interp_clamped(xg, yg, x):
    """Piecewise-linear y(x) on the sorted grid xg, clamped to the end values
    outside it (_interp1d_vec, src/FFAG_bucket.py:9-24: the interval from
    searchsorted(xg, x) - 1, y0 + (y1 - y0)(x - x0)/(x1 - x0))."""
    x = np.asarray(x, np.float64)
    j = np.clip(np.searchsorted(xg, x) - 1, 0, len(xg) - 2)
    x0, x1, y0, y1 = xg[j], xg[j + 1], yg[j], yg[j + 1]
    out = y0 + (y1 - y0) * (x - x0) / (x1 - x0)
    out = np.where(x <= xg[0], yg[0], out)
    return np.where(x >= xg[-1], yg[-1], out)


def _linear_extrap(X, Y, xi):
    """Linear interpolation with linear extrapolation from the end intervals
    (linear_interpolation_vect / find_two_points_non_uniform_vect,
    src/FFAG_MathTools.py:59-82, 162-173)."""
    xi = np.asarray(xi, np.float64)
    right = np.searchsorted(X, xi, side="right")
    i0 = np.clip(right - 1, 0, len(X) - 2)
    i0 = np.where(right > len(X) - 1, len(X) - 2, i0)
    x0, x1, y0, y1 = X[i0], X[i0 + 1], Y[i0], Y[i0 + 1]
    return y0 + (xi - x0) / (x1 - x0) * (y1 - y0)


class FFAG_bucket:
    """The RF bucket of one synchronous energy; the reference's constructor
    arguments (fi0 in degrees)."""

    def __init__(self, Bmapfoldname, Ek0=300.0, fi0=30.0, U0=100e3, step_t=20e-9, step_N=15000):
        data = np.loadtxt(os.path.join(Bmapfoldname, "resultsSEO", "SEO_ini.txt"), skiprows=2)
        Ek_seo = data[:, 1].astype(np.float64)
        f_seo = data[:, 4].astype(np.float64)
        T_seo = 1.0 / f_seo
        order = np.argsort(Ek_seo)
        self.Ek_seo, self.f_seo, self.T_seo = Ek_seo, f_seo, T_seo
        self.Ek_grid = np.ascontiguousarray(Ek_seo[order])
        self.T_grid = np.ascontiguousarray(T_seo[order])
        self.E0 = float(Ek0)
        self.fi0 = float(np.deg2rad(fi0))
        self.U0 = float(U0)
        self.step_t = float(step_t)
        self.max_stepsN = int(step_N)
        self.Tc = float(_linear_extrap(Ek_seo, T_seo, np.array([self.E0]))[0])
        self.w0 = float(_linear_extrap(Ek_seo, f_seo, np.array([self.E0]))[0] * 2 * np.pi)
        # starting points: a ring round the unstable fixed point, and the centre line
        phi_s = self.fi0
        phi_u = np.pi - phi_s
        self.zd_u = (phi_u - phi_s) / self.w0
        th = np.linspace(0, 2 * np.pi, 20, endpoint=False)
        self.X_sep = np.column_stack((self.zd_u + 5.0e-9 * np.cos(th), 0.5 * np.sin(th)))
        z_ns = np.linspace(-0.8 * abs(self.zd_u) * 1e9, 0.0, 20)
        self.X_center = np.column_stack((z_ns * 1e-9, np.zeros(20)))
        self.X_in = np.vstack([self.X_sep, self.X_center])
        self.tr_fwd = self.rk4_solve_dt(self.dynamic, 0.0, self.X_in)
        self.stable_fwd, _ = self.classify_stability(self.tr_fwd)
        self.tr_rev = self.rk4_solve_dt(self.dynamic_neg, 0.0, self.X_in)
        self.stable_rev, _ = self.classify_stability(self.tr_rev)
        self.x_min_plot, self.x_max_plot, self.y_min_plot, self.y_max_plot = self._axes_limits()
        self.x_min_sample, self.x_max_sample, self.y_min_sample, self.y_max_sample = self._sample_limits()
        self.q_grid = self.p_grid = self.Hq_rel = self.Hp_rel = None
        self.H00 = self.H_map = self.H_sep = None
        self._H_center = self._L_center = None

    # --------------------------------------------------------- the flow
    def dynamic(self, t, X):
        zd, dEk = X[:, 0], X[:, 1]
        T = _interp_clamped(self.Ek_grid, self.T_grid, self.E0 + dEk)
        out = np.empty_like(X)
        out[:, 0] = -(self.Tc - T) / self.Tc
        out[:, 1] = (self.U0 * (np.sin(self.fi0 + self.w0 * zd) - np.sin(self.fi0)) / self.Tc) / 1e6
        return out

    def dynamic_neg(self, t, X):
        return -self.dynamic(t, X)

    def rk4_step(self, func, t, r, h):
        k1 = h * func(t, r)
        k2 = h * func(t + 0.5 * h, r + 0.5 * k1)
        k3 = h * func(t + 0.5 * h, r + 0.5 * k2)
        k4 = h * func(t + h, r + k3)
        return (k1 + 2 * k2 + 2 * k3 + k4) / 6

    def rk4_solve_dt(self, func, t_start, r_start):
        """(step_N, points, 3): t, zd, dEk before each step."""
        r = np.array(r_start, np.float64)
        tr = np.zeros((self.max_stepsN, r.shape[0], 3))
        t = float(t_start)
        for i in range(self.max_stepsN):
            tr[i, :, 0] = t
            tr[i, :, 1:] = r
            r = r + self.rk4_step(func, t, r, self.step_t)
            t += self.step_t
        return tr

    def classify_stability(self, tr, growth_tol=0.2, frac_split=0.5):
        """Stable: |w0 zd| < pi throughout and neither the phase nor the energy
        amplitude of the second part exceeds the first's by more than
        growth_tol (classify_stability, src/FFAG_bucket.py:168-195)."""
        steps, P, _ = tr.shape
        split = max(4, int(steps * frac_split))
        stable = np.ones(P, dtype=bool)
        why = [""] * P
        for k in range(P):
            zd, dE = tr[:, k, 1], tr[:, k, 2]
            ph = ((self.fi0 + self.w0 * zd - self.fi0) + np.pi) % (2 * np.pi) - np.pi
            if np.any(np.abs(self.w0 * zd) >= np.pi):
                stable[k], why[k] = False, "crossed |phi - fi0| = pi"
                continue
            a1 = max(np.max(np.abs(ph[:split])), 1e-12)
            a2 = np.max(np.abs(ph[split:])) if split < steps else a1
            e1 = max(np.max(np.abs(dE[:split])), 1e-12)
            e2 = np.max(np.abs(dE[split:])) if split < steps else e1
            if a2 / a1 > 1.0 + growth_tol or e2 / e1 > 1.0 + growth_tol:
                stable[k], why[k] = False, "amplitude growth"
            else:
                why[k] = "bounded"
        return stable, why

    def _sample_limits(self):
        tmin = emin = np.inf
        tmax = emax = -np.inf
        for tr, mask in ((self.tr_fwd, self.stable_fwd), (self.tr_rev, self.stable_rev)):
            for k in range(self.X_in.shape[0]):
                if mask[k]:
                    x = tr[:, k, 1] * 1e9
                    y = tr[:, k, 2] + self.E0
                    tmin, tmax = min(tmin, x.min()), max(tmax, x.max())
                    emin, emax = min(emin, y.min()), max(emax, y.max())
        return tmin, tmax, emin, emax

    def _axes_limits(self):
        zs, es = [], []
        for tr, mask in ((self.tr_fwd, self.stable_fwd), (self.tr_rev, self.stable_rev)):
            if mask.any():
                zs.append((tr[:, mask, 1] * 1e9).ravel())
                es.append((tr[:, mask, 2] + self.E0).ravel())
        if not zs:
            return -20.0, 20.0, self.E0 - 2.0, self.E0 + 2.0
        z, e = np.concatenate(zs), np.concatenate(es)
        x0, x1, y0, y1 = z.min(), z.max(), e.min(), e.max()
        px = 0.10 * (x1 - x0) if x1 > x0 else 1.0
        py = 0.10 * (y1 - y0) if y1 > y0 else 0.1
        return x0 - px, x1 + px, y0 - py, y1 + py

    # --------------------------------------------------------- H
    @staticmethod
    def _cumtrapz(y, x):
        acc = np.zeros_like(x)
        for i in range(1, x.size):
            acc[i] = acc[i - 1] + 0.5 * (y[i - 1] + y[i]) * (x[i] - x[i - 1])
        return acc

    def A_of_p(self, p):
        T = np.interp(self.E0 + p, self.Ek_grid, self.T_grid, left=self.T_grid[0], right=self.T_grid[-1])
        return -(self.Tc - T) / self.Tc

    def B_of_q(self, q):
        return (self.U0 * (np.sin(self.fi0 + self.w0 * q) - np.sin(self.fi0)) / self.Tc) / 1e6

    def build_H(self, Nq=241, Np=241):
        """H on an Nq x Np grid of the plot box, relative to H at the
        synchronous point; H_sep at the unstable fixed point (build_H,
        src/FFAG_bucket.py:253-281)."""
        x_ns = np.linspace(self.x_min_plot, self.x_max_plot, Nq)
        y_Ek = np.linspace(self.y_min_plot, self.y_max_plot, Np)
        self.q_grid, self.p_grid = x_ns * 1e-9, y_Ek - self.E0
        self.Hp_rel = self._cumtrapz(self.A_of_p(self.p_grid), self.p_grid)
        self.Hq_rel = -self._cumtrapz(self.B_of_q(self.q_grid), self.q_grid)
        Hq0 = np.interp(0.0, self.q_grid, self.Hq_rel, left=np.nan, right=np.nan)
        Hp0 = np.interp(0.0, self.p_grid, self.Hp_rel, left=np.nan, right=np.nan)
        if np.isnan(Hq0):
            Hq0 = self.Hq_rel[0] if abs(self.q_grid[0]) < abs(self.q_grid[-1]) else self.Hq_rel[-1]
        if np.isnan(Hp0):
            Hp0 = self.Hp_rel[0] if abs(self.p_grid[0]) < abs(self.p_grid[-1]) else self.Hp_rel[-1]
        self.H00 = Hq0 + Hp0
        self.H_map = self.Hq_rel[:, None] + self.Hp_rel[None, :] - self.H00
        hq = np.interp(self.zd_u, self.q_grid, self.Hq_rel, left=self.Hq_rel[0], right=self.Hq_rel[-1])
        hp = np.interp(0.0, self.p_grid, self.Hp_rel, left=self.Hp_rel[0], right=self.Hp_rel[-1])
        self.H_sep = (hq + hp) - self.H00

    def H_at(self, q, p):
        hq = np.interp(q, self.q_grid, self.Hq_rel, left=self.Hq_rel[0], right=self.Hq_rel[-1])
        hp = np.interp(p, self.p_grid, self.Hp_rel, left=self.Hp_rel[0], right=self.Hp_rel[-1])
        return (hq + hp) - self.H00

    def compute_center_H_vs_span(self):
        """H of each stable centre-line trajectory and its time span [ns]
        (the smaller of the forward and backward spans), sorted by H."""
        n0 = self.X_sep.shape[0]
        Hc = self.H_at(self.X_center[:, 0], self.X_center[:, 1])
        H, L = [], []
        for k in range(self.X_center.shape[0]):
            pid = n0 + k
            spans = [float(np.ptp(tr[:, pid, 1] * 1e9)) for tr, st in
                     ((self.tr_fwd, self.stable_fwd), (self.tr_rev, self.stable_rev)) if st[pid]]
            if spans:
                H.append(float(Hc[k]))
                L.append(min(spans))
        if not H:
            raise RuntimeError("no stable centre-line trajectory to relate H to a bunch length")
        o = np.argsort(np.array(H))
        self._H_center, self._L_center = np.array(H)[o], np.array(L)[o]
        return self._H_center, self._L_center

    def threshold(self, L_target_ns):
        """H of the centre-line trajectory whose span is L_target_ns (clipped
        to the spans found), by linear interpolation in the span."""
        if self.H_map is None:
            self.build_H()
        if self._H_center is None:
            self.compute_center_H_vs_span()
        H, L = self._H_center, self._L_center
        Lu = float(np.clip(L_target_ns, L.min(), L.max()))
        o = np.argsort(L)
        return float(_linear_extrap(L[o], H[o], np.array([Lu]))[0])

    def scatter_filter_by_span(self, N_demo, L_target_ns, show=False, rng=None):
        """N_demo points (t [ns], Ek [MeV]) uniform in the sampling box with
        H >= the threshold of L_target_ns; returns (t, Ek, H_thr)."""
        rng = rng if rng is not None else np.random.default_rng()
        H_thr = self.threshold(L_target_ns)
        acc = np.zeros((0, 2))
        while acc.shape[0] < N_demo:
            x = rng.uniform(self.x_min_sample, self.x_max_sample, size=int(N_demo) * 10)
            y = rng.uniform(self.y_min_sample, self.y_max_sample, size=int(N_demo) * 10)
            keep = self.H_at(x * 1e-9, y - self.E0) >= H_thr
            acc = np.vstack((acc, np.column_stack((x[keep], y[keep]))))
        acc = acc[:N_demo]
        return acc[:, 0], acc[:, 1], H_thr
