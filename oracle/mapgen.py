"""CPU restatement of the reference's z-Taylor map generator.

TEST INFRASTRUCTURE ONLY: the checker for pyffa_b200.mapgen (tests/ only).

Restates Generate_Bmaps / Generate_Bmaps_MultiProcess
(src/FFAG_HighOrder.py:828-998) term by term and in the same evaluation
order, with numpy float64:

* the mid-plane field is B0(r, th) = A(r) G(th - s(r)), A(r) = a r^k
  (recursive_nth_derivative, :448-487), G the sum of sigmoid-pair flutter
  shapes (shape_function / shape_function_nth_derivative, :246-350) whose
  derivatives are polynomials in the sigmoid (sigmoid_nth_derivative,
  :212-244);
* the spiral shift is applied by rolling the sampled G by
  int(s(r) / dth) grid steps (shift_function, :393-398);
* r-derivatives of G(th - s(r)) follow the chain-rule term lists of
  calculate_first_derivative / merge_terms / dGn_dnR_Vals (:11-131);
* the Laplacian powers are kept as (m, n, k, a) rows meaning
  a d^m/dr^m d^n/dth^n B / r^k (apply_*_derivative, apply_laplacian_combined,
  merge_similar_terms, :524-655), evaluated by Polar_Laplace_Vals (:747-769);
* order n: Bz_n = (-1)^n/(2n)! L^n B0 / MeanF, Br_n = (-1)^n/(2n+1)!
  d_r L^n B0 / MeanF, Bfi_n = (-1)^n/(2n+1)! / r d_th L^n B0 / MeanF, MeanF
  the mean of G over the sector at that r (:873-896).  The 1/MeanF factor is
  the reference's: the tables it writes for a scaling map are the exact
  expansion divided by the sector mean of the flutter.

Pinned against the reference's own output on two lattices
(tests/golden/golden_mapgen.npz, tests/golden/make_golden.py --mapgen).
"""
from __future__ import annotations

from math import factorial

import numpy as np
from scipy.special import binom


def calculate_s(r_axis, s0, alpha_deg):
    """Spiral azimuth s(r) by the reference's running sum (:400-421)."""
    s = np.zeros_like(r_axis)
    s[0] = s0
    t = np.tan(np.deg2rad(alpha_deg))
    for i in range(1, len(r_axis)):
        s[i] = s[i - 1] + t / r_axis[i] * (r_axis[i] - r_axis[i - 1])
    return s


def convex_params(bmap: dict):
    """(x0, x1, W0, (|pol|, sign)) per magnet, BmapParams_to_ConvexParams (:1001-1030)."""
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


def _sigmoid(x, x0, k):
    return 1 / (1 + np.exp(-k * (x - x0)))


def _sigmoid_deriv(x0, k, order, x):
    """sigma^(order) as a polynomial in sigma (:212-244)."""
    s = _sigmoid(x, x0, k)
    if order == 0:
        return s
    base = np.array([-k, k, 0], dtype=np.float64)
    c = base
    for _ in range(order - 1):
        n = len(c) - 1
        d = np.array([c[i] * (n - i) for i in range(n)], dtype=np.float64)
        c = np.convolve(d, base).astype(np.float64)
    out = np.zeros_like(s)
    for coef in c:
        out = out * s + coef
    return out


def _binom_int(n, k):
    return factorial(n) // (factorial(k) * factorial(n - k))


def _shape(x, p):
    x0, x1, W0, y01 = p
    yc = y01[1] * np.abs(y01[0])
    k = 16 / W0
    return 0 + (yc - 0) * _sigmoid(x, x0, k) * _sigmoid(x, x1, -k)


def _shape_deriv(x, p, n):
    x0, x1, W0, y01 = p
    yc = y01[1] * np.abs(y01[0])
    k = 16 / W0
    res = np.zeros_like(x)
    for i in range(n + 1):
        res += _binom_int(n, i) * _sigmoid_deriv(x0, k, i, x) * _sigmoid_deriv(x1, -k, n - i, x)
    return (yc - 0) * res


def flutter(x, convex, n):
    """(G, G^(n)) on the grid (generate_shapes_with_derivatives, :372-391)."""
    tot = np.zeros_like(x)
    if n == 0:
        for p in convex:
            tot += _shape(x, p)
        return tot, tot
    der = np.zeros_like(x)
    for p in convex:
        tot += _shape(x, p)
        der += _shape_deriv(x, p, n)
    return tot, der


def _roll(x, y, dx):
    return np.roll(y, int(dx / (x[1] - x[0])))


def chain_terms(order):
    """d^order/dr^order of G(th - s(r)) as [p, coef, e0, e1, ...] rows:
    coef * G^(p) * prod_i (s^(i))^(e_i) (:11-91)."""
    cur = [np.array([0.0, 1.0, 0.0])]
    for _ in range(order):
        nxt = []
        for t in cur:
            p, c, m = t[0], t[1], t[2:]
            mm = np.copy(m)
            if len(mm) > 1:
                mm[1] += 1
            else:
                mm = np.append(mm, 1)
            nxt.append(np.concatenate(([p + 1, -c], mm)))
            for i in range(len(m)):
                if m[i] > 0:
                    mm = np.copy(m)
                    mm[i] -= 1
                    if i + 1 < len(mm):
                        mm[i + 1] += 1
                    else:
                        mm = np.append(mm, 1)
                    nxt.append(np.concatenate(([p, c * m[i]], mm)))
        merged = {}
        for t in nxt:
            key = (t[0], tuple(t[2:]))
            merged[key] = merged.get(key, 0.0) + t[1]
        cur = [np.concatenate(([p, c], np.array(m))) for (p, m), c in merged.items() if c != 0]
    return cur


def dG_dr(order, fi, convex, sfit, r, order_plus=0):
    """dGn_dnR_Vals (:94-131)."""
    sr = sfit(r)
    out = np.zeros_like(fi)
    for t in chain_terms(order):
        p, c, m = np.int64(t[0]), t[1], t[2:]
        g = _roll(fi, flutter(fi, convex, p + order_plus)[1], sr)
        S = 1.0
        for i, e in enumerate(m):
            S *= sfit.deriv(m=i)(r) ** e
        out += g * c * S
    return out


def A_deriv(a, k, n, r):
    """recursive_nth_derivative for the power law (:448-470)."""
    kv = np.append(np.arange(k, k - n, -1), 1)
    return a * np.prod(kv) * r ** (k - n)


def _merge(rows):
    d = {}
    for m, n, k, a in rows:
        key = (m, n, k)
        d[key] = d.get(key, 0) + a
    return np.array([[*key, v] for key, v in d.items()])


def _dr(rows):
    out = []
    for m, n, k, a in rows:
        m, n, k, a = int(m), int(n), int(k), int(a)
        out.append([m + 1, n, k, a])
        if k != 0:
            out.append([m, n, k + 1, -a * k])
    return np.array(out)


def _dth(rows):
    return np.array([[int(m), int(n) + 1, int(k), int(a)] for m, n, k, a in rows])


def _rpow(rows, p):
    return np.array([[int(m), int(n), int(k) + p, int(a)] for m, n, k, a in rows])


def _laplacian(rows):
    return np.vstack((_dr(_dr(rows)), _rpow(_dr(rows), 1), _rpow(_dth(_dth(rows)), 2)))


def _polar_laplace(rows, r, fi, convex, sfit, ak):
    res = np.zeros_like(fi)
    for row in rows:
        nr, mth, kk, a0 = row[0], row[1], row[2], row[3]
        dB = 0
        for i in range(0, int(nr) + 1):
            dB += binom(nr, i) * dG_dr(i, fi, convex, sfit, r, order_plus=mth) * A_deriv(ak[0], ak[1], nr - i, r)
        res += dB * (a0 / r ** kk)
    return res


def generate_bmaps(max_order, r_axis, fi_axis, convex, sfit, ak):
    """(Br, Bz, Bfi) lists of (n_r, n_th) tables for orders 0..max_order."""
    Br, Bz, Bfi = [], [], []
    L = np.array([[0, 0, 0, 1]])
    for n in range(max_order + 1):
        Lr = _dr(L)
        Lf = _dth(L)
        c1 = (-1) ** n / factorial(2 * n + 1)
        c0 = (-1) ** n / factorial(2 * n)
        L, Lr, Lf = _merge(L), _merge(Lr), _merge(Lf)
        bz = np.zeros((len(r_axis), len(fi_axis)))
        br = np.zeros_like(bz)
        bfi = np.zeros_like(bz)
        for i, r in enumerate(r_axis):
            meanF = np.mean(dG_dr(0, fi_axis, convex, sfit, r))
            bz[i] = c0 * _polar_laplace(L, r, fi_axis, convex, sfit, ak) / meanF
            br[i] = c1 * _polar_laplace(Lr, r, fi_axis, convex, sfit, ak) / meanF
            bfi[i] = c1 / r * _polar_laplace(Lf, r, fi_axis, convex, sfit, ak) / meanF
        Br.append(br)
        Bz.append(bz)
        Bfi.append(bfi)
        L = _laplacian(L)
    return Br, Bz, Bfi


def axes(bmap: dict):
    """r and th axes of main_Bmap (examples/main_Bmap.py:40-45)."""
    rmin, rmax, rstep = bmap["rmin_max_step_m"]
    n_r = int((rmax - rmin) / rstep) + 1
    n_fi = int((np.pi * 2 / bmap["NSector"] - 0.0) / bmap["theta_step_rad"]) + 1
    return np.linspace(rmin, rmax, n_r), np.linspace(0, np.pi * 2 / bmap["NSector"], n_fi)
