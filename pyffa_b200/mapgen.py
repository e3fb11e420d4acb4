"""z-Taylor map generation on the GPU.

Drop-in for the reference's offline map builder: Generate_Bmaps /
Generate_Bmaps_MultiProcess (src/FFAG_HighOrder.py:828-998) with the same
arguments and the same (Br, Bz, Bfi) lists of (n_r, n_theta) float64 tables
per order, and main_Bmap (examples/main_Bmap.py:17-75), which writes
``Br/Bz/Bfi_order_{n}.npz`` (keys ``*_Taylor_coeff``) next to the lattice
JSON.

The reference's result for order n is, per radius r and azimuth th,

    Bz_n  = (-1)^n / (2n)!     L^n B0 / MeanF
    Br_n  = (-1)^n / (2n+1)!   d_r L^n B0 / MeanF
    Bfi_n = (-1)^n / (2n+1)! / r d_th L^n B0 / MeanF

with L the polar Laplacian d_rr + d_r / r + d_thth / r^2, B0 = a r^k G(th - s(r)),
G the flutter (sum of sigmoid pairs), MeanF the sector mean of G (the
reference divides every order by it, the order-0 table included).  Each L^n
term a d_r^m d_th^q B0 / r^kk expands (Leibniz in r, chain rule through
s(r)) into products of an r-only factor and one flutter derivative G^(p); so
every entry is sum_p w_p(r) G^(p)(th - shift(r)), the spiral shift being the
reference's integer roll of the sampled G by int(s(r) / dth) nodes
(shift_function, src/FFAG_HighOrder.py:393-398).  This module forms the
weights w (tiny, vectorised over r); libffa_cuda.so evaluates G^(p) on the
theta grid and writes the tables (ffa_mapgen).
"""
from __future__ import annotations

import ctypes
import json
import os
from math import comb, factorial

import numpy as np
from numpy.polynomial import Polynomial

from . import _lib

# ---------------------------------------------------------------- lattice


def calculate_s(r_axis, s0, alpha_deg):
    """Spiral azimuth s(r) as the reference's running sum
    (calculate_s, src/FFAG_HighOrder.py:400-421)."""
    s = np.zeros_like(np.asarray(r_axis, dtype=np.float64))
    s[0] = s0
    t = np.tan(np.deg2rad(alpha_deg))
    for i in range(1, len(r_axis)):
        s[i] = s[i - 1] + t / r_axis[i] * (r_axis[i] - r_axis[i - 1])
    return s


def BmapParams_to_ConvexParams(bmap: dict):
    """(x0, x1, W0, (|polarity|, sign)) per magnet in rad
    (src/FFAG_HighOrder.py:1001-1030)."""
    out = []
    total = 360.0 / bmap["NSector"]
    start = 0
    for interval, pol, fringe in zip(bmap["interval_1"], bmap["positive_or_negative_1"], bmap["fringe_width_1"]):
        if pol == 0:
            start += interval * total
            continue
        end = start + interval * total
        out.append((np.deg2rad(start), np.deg2rad(end), np.deg2rad((end - start) * fringe),
                    (abs(pol), 1 if pol > 0 else -1)))
        start = end
    return out


def map_axes(bmap: dict):
    """r and theta axes of main_Bmap (examples/main_Bmap.py:40-45)."""
    rmin, rmax, rstep = bmap["rmin_max_step_m"]
    n_r = int((rmax - rmin) / rstep) + 1
    n_fi = int((np.pi * 2 / bmap["NSector"] - 0.0) / bmap["theta_step_rad"]) + 1
    return np.linspace(rmin, rmax, n_r), np.linspace(0, np.pi * 2 / bmap["NSector"], n_fi)


# ---------------------------------------------------------- term algebra


def _chain(order: int) -> dict:
    """d^order/dr^order of G(th - s(r)) as {(p, exps): coef}: coef G^(p)
    prod_l (s^(l))^exps[l] (the chain rule of calculate_first_derivative,
    src/FFAG_HighOrder.py:11-46; exps without trailing zeros)."""
    terms = {(0, ()): 1}
    for _ in range(order):
        nxt: dict = {}

        def add(key, c):
            p, e = key
            e = tuple(e)
            while e and e[-1] == 0:
                e = e[:-1]
            nxt[(p, e)] = nxt.get((p, e), 0) + c

        for (p, e), c in terms.items():
            e = list(e) + [0, 0]
            # d/dr G^(p)(th - s) = -G^(p+1) s'
            e1 = list(e)
            e1[1] += 1
            add((p + 1, e1), -c)
            # d/dr (s^(l))^m = m (s^(l))^(m-1) s^(l+1)
            for l, m in enumerate(e):
                if m > 0:
                    e2 = list(e)
                    e2[l] -= 1
                    e2[l + 1] += 1
                    add((p, e2), c * m)
        terms = {k: v for k, v in nxt.items() if v != 0}
    return terms


def _dr(rows: dict) -> dict:
    """d/dr of sum a d_r^m d_th^q B / r^kk (apply_r_derivative, :545-566)."""
    out: dict = {}
    for (m, q, kk), a in rows.items():
        out[(m + 1, q, kk)] = out.get((m + 1, q, kk), 0) + a
        if kk != 0:
            out[(m, q, kk + 1)] = out.get((m, q, kk + 1), 0) - a * kk
    return out


def _dth(rows: dict) -> dict:
    out: dict = {}
    for (m, q, kk), a in rows.items():
        out[(m, q + 1, kk)] = out.get((m, q + 1, kk), 0) + a
    return out


def _laplacian(rows: dict) -> dict:
    """d_rr + d_r / r + d_thth / r^2 (apply_laplacian_combined, :635-655)."""
    out: dict = {}
    for part, dk in ((_dr(_dr(rows)), 0), (_dr(rows), 1), (_dth(_dth(rows)), 2)):
        for (m, q, kk), a in part.items():
            out[(m, q, kk + dk)] = out.get((m, q, kk + dk), 0) + a
    return out


def _a_deriv(a, k, n, r):
    """n-th derivative of a r^k (recursive_nth_derivative, :448-470)."""
    c = a * float(np.prod(np.append(np.arange(k, k - n, -1), 1)))
    return c * r ** (k - n)


def n_derivatives(max_order: int) -> int:
    return 2 * max_order + 2


def weights(max_order, r_axis, ak, sfit):
    """(3, max_order+1, n_r, n_deriv) weights of G^(p): Bz, Br, Bfi, before
    the division by the sector mean of G."""
    r = np.asarray(r_axis, dtype=np.float64)
    a, k = float(ak[0]), float(ak[1])
    P = n_derivatives(max_order)
    W = np.zeros((3, max_order + 1, len(r), P))
    sder = [sfit.deriv(m=l)(r) for l in range(2 * max_order + 2)]
    chains = [_chain(i) for i in range(2 * max_order + 2)]
    L = {(0, 0, 0): 1}
    for n in range(max_order + 1):
        c0 = (-1) ** n / factorial(2 * n)
        c1 = (-1) ** n / factorial(2 * n + 1)
        for comp, rows, const in ((0, L, c0 * np.ones_like(r)), (1, _dr(L), c1 * np.ones_like(r)),
                                  (2, _dth(L), c1 / r)):
            for (m, q, kk), a0 in rows.items():
                if a0 == 0:
                    continue
                fac = const * (a0 / r ** kk)
                for i in range(m + 1):
                    ai = comb(m, i) * _a_deriv(a, k, m - i, r)
                    for (p, e), c in chains[i].items():
                        S = np.ones_like(r)
                        for l, ex in enumerate(e):
                            if ex:
                                S = S * sder[l] ** ex
                        W[comp, n, :, p + q] += fac * ai * c * S
        L = _laplacian(L)
    return W


def sigmoid_polys(k: float, n_deriv: int) -> np.ndarray:
    """(n_deriv, n_deriv+1): row i = coefficients (highest first, i+2 used) of
    the i-th derivative of the sigmoid of steepness k as a polynomial in the
    sigmoid (sigmoid_nth_derivative, src/FFAG_HighOrder.py:212-244; row 0 is
    the sigmoid itself)."""
    out = np.zeros((n_deriv, n_deriv + 1))
    out[0, :2] = [1.0, 0.0]
    base = np.array([-k, k, 0], dtype=np.float64)
    c = base
    for i in range(1, n_deriv):
        out[i, :len(c)] = c
        n = len(c) - 1
        d = np.array([c[j] * (n - j) for j in range(n)], dtype=np.float64)
        c = np.convolve(d, base).astype(np.float64)
    return out


# ---------------------------------------------------------------- driver


class MapgenPlan:
    """Host weights and device inputs of one map build; run() launches the
    build (ffa_mapgen) and returns the (3, max_order+1, n_r, n_theta) float64
    tables (Bz, Br, Bfi) on the device.  The plan keeps every device buffer
    the launch reads alive."""

    def __init__(self, max_order, r_axis, fi_axis_rad, convex_params, sfit, ak, device=None):
        import torch
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        r = np.asarray(r_axis, dtype=np.float64)
        fi = np.asarray(fi_axis_rad, dtype=np.float64)
        if len(convex_params) > _lib.MAX_SEG:
            raise ValueError(f"at most {_lib.MAX_SEG} flutter magnets")
        P = n_derivatives(max_order)
        if P > _lib.MAPGEN_MAX_DERIV:
            raise ValueError(f"max_order {max_order} needs {P} flutter derivatives "
                             f"(limit {_lib.MAPGEN_MAX_DERIV})")
        W = weights(max_order, r, ak, sfit)
        dth = fi[1] - fi[0]
        shift = np.array([int(sfit(x) / dth) for x in r], dtype=np.int32)
        polys = np.zeros((len(convex_params), 2, P, P + 1))
        d = _lib.MapgenDesc()
        d.n_seg, d.n_deriv, d.n_orders = len(convex_params), P, max_order + 1
        d.n_r, d.n_theta = len(r), len(fi)
        for j, (x0, x1, W0, y01) in enumerate(convex_params):
            k = 16 / W0
            d.seg_x0[j], d.seg_x1[j], d.seg_k[j] = x0, x1, k
            d.seg_y[j] = y01[1] * np.abs(y01[0])
            polys[j, 0] = sigmoid_polys(k, P)
            polys[j, 1] = sigmoid_polys(-k, P)
        f64 = dict(dtype=torch.float64, device=dev)
        self._in = [torch.from_numpy(np.ascontiguousarray(x).reshape(-1)).to(dev)
                    for x in (polys, fi, W, shift)]
        self.gder = torch.empty(P * len(fi), **f64)
        self.gmean = torch.empty(1, **f64)
        self.tables = torch.empty((3, max_order + 1, len(r), len(fi)), **f64)
        d.sig_poly, d.theta, d.weights, d.shift = (t.data_ptr() for t in self._in)
        d.gder, d.gmean = self.gder.data_ptr(), self.gmean.data_ptr()
        d.bz, d.br, d.bfi = (self.tables[c].data_ptr() for c in range(3))
        self.desc = d

    def run(self):
        import torch
        stream = torch.cuda.current_stream(self.device)
        _lib.check(_lib.lib().ffa_mapgen(ctypes.byref(self.desc), stream.cuda_stream), "ffa_mapgen")
        return self.tables


def generate_device(max_order, r_axis, fi_axis_rad, convex_params, sfit, ak, device=None):
    """The tables on the GPU: (3, max_order+1, n_r, n_theta) float64 (Bz, Br, Bfi)."""
    import torch
    plan = MapgenPlan(max_order, r_axis, fi_axis_rad, convex_params, sfit, ak, device)
    out = plan.run()
    torch.cuda.current_stream(plan.device).synchronize()   # the plan's inputs are freed on return
    return out


def Generate_Bmaps(MaxOrder, r_axis, fi_axis_rad, convex_paras, s_values_FitCoef_rad, BzR_coef_k):
    """Reference signature (src/FFAG_HighOrder.py:828): returns the lists
    (Br, Bz, Bfi) of (n_r, n_theta) numpy tables for orders 0..MaxOrder."""
    t = generate_device(MaxOrder, r_axis, fi_axis_rad, convex_paras, s_values_FitCoef_rad, BzR_coef_k).cpu().numpy()
    return [t[1, n] for n in range(MaxOrder + 1)], [t[0, n] for n in range(MaxOrder + 1)], \
        [t[2, n] for n in range(MaxOrder + 1)]


Generate_Bmaps_MultiProcess = Generate_Bmaps


def main_Bmap(json_path: str) -> str:
    """examples/main_Bmap.py: reads the lattice JSON, writes the order tables
    and the JSON with the sector-mean field (Bmap.Bmean, Bmap.r_axis, which the
    closed-orbit search starts from) into config.folder (relative to the
    JSON), and returns that folder."""
    from .fields import FFAG_Bfield_analytical
    json_dir = os.path.dirname(os.path.abspath(json_path))
    with open(json_path) as f:
        cfg = json.load(f)
    bmap = cfg["Bmap"]
    folder = cfg["config"]["folder"]
    out_dir = folder if os.path.isabs(folder) else os.path.join(json_dir, folder)
    os.makedirs(out_dir, exist_ok=True)
    FFAG_Bfield_analytical(json_path, 0, AddNumricalMap=False).UpdataConfig(out_dir)
    r, fi = map_axes(bmap)
    s = calculate_s(r, 0.0, bmap["SpiralAngle_deg"])
    sfit = Polynomial.fit(r, s, 5)
    Br, Bz, Bfi = Generate_Bmaps(cfg["config"]["expand_order"], r, fi, BmapParams_to_ConvexParams(bmap), sfit,
                                 bmap["coefficients_tupel"])
    for n in range(len(Br)):
        np.savez(os.path.join(out_dir, f"Br_order_{n}.npz"), Br_Taylor_coeff=Br[n])
        np.savez(os.path.join(out_dir, f"Bz_order_{n}.npz"), Bz_Taylor_coeff=Bz[n])
        np.savez(os.path.join(out_dir, f"Bfi_order_{n}.npz"), Bfi_Taylor_coeff=Bfi[n])
    return out_dir
