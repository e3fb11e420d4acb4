"""Seeded synthetic inputs for the tracking workloads.

The reference ships no field maps, closed-orbit tables or bunches, and its
bunch generator is unseeded, so every workload here is generated from a
seed: the 12-sector scaling-FFAG lattice, its z-Taylor coefficient tables,
an RF frequency-curve file in the reference's 4-column format, closed-orbit
tables for the space-charge step, and 6D Gaussian / KV bunches in the
reference's p-format (r, pr, z, pz, fi, Ek[MeV], inj_t[ns], flags, ...).

The z-Taylor tables are the exact expansion of the analytic field for a
zero spiral angle: with Bz(z=0) = B0 r^k F(theta),
    Bz = sum_n a_n z^(2n),  a_n = B0 r^(k-2n) P_n(theta),
    P_0 = F,  P_(n+1) = -((k-2n)^2 P_n + P_n'') / ((2n+2)(2n+1)),
    Br = sum_n d(a_n)/dr z^(2n+1)/(2n+1),  Bfi = sum_n (1/r) d(a_n)/dtheta z^(2n+1)/(2n+1),
so curl B = 0 and div B = 0 hold order by order.  The flutter derivatives
F^(m) are taken analytically from the logistic fringes.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from .constants import C_LIGHT, E0_J, E0_MEV, Q

# 12-sector scaling FFAG, proton 300 MeV, k = 7.6, F-D cell with sector
# fractions (0.25, 0.3125, 0.09375, 0.09375, 0.25).  Two numbers differ from
# the nominal workload description, both for stability:
#  - D polarity -1.3 instead of -0.7279: with -0.7279 the cell is vertically
#    unstable (|Tr Mz|/2 = 1.39 per sector at 300 MeV);
#  - fringe widths 1.17 instead of (0.20, 0.35): edges that sharp (10-90 %
#    rise of 0.3-0.5 deg) are not resolved by 0.5-deg push steps and the
#    linear vertical motion grows without bound even at z = 0.1 mm.
# Result: Qx = 3.60, Qz = 0.78 at 300 MeV.  At 720 steps/turn the 2.8-deg
# D magnet is still coarsely sampled (betatron amplitudes diffuse slowly over
# tens of turns); at 2880 steps/turn the motion is regular.
LATTICE = {
    "NSector": 12,
    "k": 7.6,
    "interval_1": [0.25, 0.3125, 0.09375, 0.09375, 0.25],
    "positive_or_negative_1": [0, 1, 0, -1.3, 0],
    "fringe_width_1": [0, 1.17, 0, 1.17, 0],
    "SpiralAngle_deg": 0.0,
    "r_ref": 8.5,
    "Ek_ref_MeV": 300.0,
}


def momentum(Ek_MeV):
    Ek_J = np.asarray(Ek_MeV, dtype=np.float64) * 1e6 * Q
    return np.sqrt((Ek_J + E0_J) ** 2 - E0_J ** 2) / C_LIGHT


def beta_of(Ek_MeV):
    g = (np.asarray(Ek_MeV, dtype=np.float64) * 1e6 * Q + E0_J) / E0_J
    return np.sqrt(1 - 1 / g ** 2)


def logistic_derivs(u, mmax):
    """sigma(u) and its u-derivatives 0..mmax (derivative polynomials in sigma)."""
    s = 1.0 / (1.0 + np.exp(-u))
    polys = [np.polynomial.Polynomial([0.0, 1.0])]
    base = np.polynomial.Polynomial([0.0, 1.0, -1.0])  # sigma (1 - sigma)
    for _ in range(mmax):
        polys.append(polys[-1].deriv() * base)
    return [p(s) for p in polys]


def flutter_derivs(theta, convex, mmax):
    """F and its theta-derivatives 0..mmax for the reference's flutter shape
    F = sum_j y_j s1_j s2_j (GetBfields_Njit, src/FFAG_Field.py:1333-1426)."""
    out = [np.zeros_like(theta) for _ in range(mmax + 1)]
    for x0, x1, W0, y01, y02 in convex:
        k = 16.0 / W0
        y = y02 * abs(y01)
        d1 = logistic_derivs(k * (theta - x0), mmax)
        d2 = logistic_derivs(-k * (theta - x1), mmax)
        for m in range(mmax + 1):
            acc = np.zeros_like(theta)
            for j in range(m + 1):
                acc += math.comb(m, j) * (k ** j * d1[j]) * ((-k) ** (m - j) * d2[m - j])
            out[m] += y * acc
    return out


def lattice_bmap(B0=None, r_range=(8.0, 9.3, 0.001), theta_step_deg=0.005, lattice=LATTICE) -> dict:
    """config_Bmap.json content for the lattice (reference key names)."""
    from .fields import convex_params
    bm = {
        "NSector": lattice["NSector"],
        "rmin_max_step_m": list(r_range),
        "SpiralAngle_deg": lattice["SpiralAngle_deg"],
        "theta_step_rad": float(np.deg2rad(theta_step_deg)),
        "interval_1": lattice["interval_1"],
        "positive_or_negative_1": lattice["positive_or_negative_1"],
        "fringe_width_1": lattice["fringe_width_1"],
        "Bmean": None,
        "r_axis": None,
    }
    if B0 is None:
        # average bending B0 r^(k+1) <F> = p/q at the reference radius
        cp = convex_params(bm)
        th = np.linspace(0, 2 * np.pi / bm["NSector"], 200001)
        Fm = flutter_derivs(th, cp, 0)[0].mean()
        brho = momentum(lattice["Ek_ref_MeV"]) / Q
        B0 = float(brho / (lattice["r_ref"] ** (lattice["k"] + 1) * Fm))
    bm["coefficients_tupel"] = [B0, lattice["k"]]
    return {"Bmap": bm, "config": {"folder": "."}}


def taylor_stacks(cfg: dict, max_order: int):
    """(Bz, Bfi, Br) coefficient stacks of shape (max_order+1, NX, NY)."""
    from .fields import FFAG_Bfield_analytical
    bm = cfg["Bmap"]
    if bm["SpiralAngle_deg"] != 0:
        raise NotImplementedError("synthetic z-Taylor tables are built for a zero spiral angle")
    f = FFAG_Bfield_analytical(config=cfg, max_order=0, AddNumricalMap=False)
    r = f.r_axis[:, None]
    th = f.fi_axis
    B0, k = f.B0, f.k_value
    P = [flutter_derivs(th, f.convex_params, 2 * max_order + 2)]  # P_0 derivatives
    # P_(n+1)^(m) = -((k-2n)^2 P_n^(m) + P_n^(m+2)) / ((2n+2)(2n+1))
    for n in range(max_order):
        prev = P[-1]
        nxt = [-((k - 2 * n) ** 2 * prev[m] + prev[m + 2]) / ((2 * n + 2) * (2 * n + 1))
               for m in range(len(prev) - 2)]
        P.append(nxt)
    shape = (max_order + 1, f.r_size, f.fi_size)
    bz, bfi, br = (np.zeros(shape) for _ in range(3))
    for n in range(max_order + 1):
        e = k - 2 * n
        rp = B0 * r ** e
        bz[n] = rp * P[n][0][None, :]
        br[n] = (B0 * e * r ** (e - 1)) * P[n][0][None, :] / (2 * n + 1)
        bfi[n] = (rp / r) * P[n][1][None, :] / (2 * n + 1)
    return bz, bfi, br


def write_bmap_folder(folder: str, max_order: int, **kw) -> str:
    """Writes config_Bmap.json and the Br/Bz/Bfi_order_n.npz files."""
    os.makedirs(folder, exist_ok=True)
    cfg = lattice_bmap(**kw)
    cfg["config"]["folder"] = folder
    path = os.path.join(folder, "config_Bmap.json")
    with open(path, "w") as f:
        json.dump(cfg, f, indent=2)
    if max_order >= 1:
        bz, bfi, br = taylor_stacks(cfg, max_order)
        for n in range(max_order + 1):
            np.savez(os.path.join(folder, f"Bz_order_{n}.npz"), Bz_Taylor_coeff=bz[n])
            np.savez(os.path.join(folder, f"Bfi_order_{n}.npz"), Bfi_Taylor_coeff=bfi[n])
            np.savez(os.path.join(folder, f"Br_order_{n}.npz"), Br_Taylor_coeff=br[n])
    return path


def orbit_radius(Ek_MeV, lattice=LATTICE):
    """Scaling-law closed-orbit radius estimate r = r_ref (p/p_ref)^(1/(k+1))."""
    p = momentum(Ek_MeV)
    pref = momentum(lattice["Ek_ref_MeV"])
    return lattice["r_ref"] * (p / pref) ** (1.0 / (lattice["k"] + 1))


def revolution_time(Ek_MeV, lattice=LATTICE):
    return 2 * np.pi * orbit_radius(Ek_MeV, lattice) / (beta_of(Ek_MeV) * C_LIGHT)


def emap_file(path: str, gap_azimuth_deg=(3.75, 183.75), rf_shift_deg=(0.0, 0.0), voltage=100e3,
              gap_width=0.2, E_range=(8.0, 9.3), harmonic=1, acc_phi_deg=30.0,
              Ek_ramp=(300.0, 310.0), ramp_turns=1000, t_start=-200e-9, npts=2001) -> str:
    """RF frequency curve in the reference's 4-column format
    (examples/main_Emap.py:752-800): time, frequency, voltage, energy, with
    the frequency following a linear energy ramp."""
    T0 = float(revolution_time(Ek_ramp[0]))
    t_end = t_start + ramp_turns * T0 * 1.05
    t = np.linspace(t_start, t_end, npts)
    frac = np.clip((t - 0.0) / (ramp_turns * T0), 0.0, 1.0)
    Ek = Ek_ramp[0] + (Ek_ramp[1] - Ek_ramp[0]) * frac
    f = harmonic / revolution_time(Ek)
    V = np.full_like(t, voltage)
    ng = len(gap_azimuth_deg)
    header = [
        "gap_model = fixed",
        f"Ngap = {ng}",
        f"acc_phi_paint = {float(acc_phi_deg)}",
        f"acc_phi_acc = {float(acc_phi_deg)}",
        f"gap_azimuth = {[float(a) for a in gap_azimuth_deg]}",
        f"rf_shift = {[float(a) for a in rf_shift_deg]}",
        f"gap_width = {float(gap_width)}",
        f"E_rmin = {float(E_range[0])}",
        f"E_rmax = {float(E_range[1])}",
        f"harmonic = {int(harmonic)}",
        f"dt_uniform = {float(t[1] - t[0]):.6e}",
        "#Time (s)        Frequency (Hz)    V0 (V)    Energy (MeV)",
    ]
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        fh.write("\n".join(header) + "\n")
        np.savetxt(fh, np.column_stack([t, f, V, Ek]), fmt="%.12e", delimiter="\t")
    return path


def spiral_emap_folder(folder: str, alpha_deg=40.0, r_ref=8.5, s_ref_deg=0.0, r_axis=(7.9, 9.3, 141),
                       pad_deg=1.0, nphi=241, sigma=0.03, gap_azimuth_deg=(3.75, 183.75), rf_shift_deg=(0.0, 0.0),
                       voltage=100e3, gap_width=0.2, harmonic=1, acc_phi_deg=30.0, Ek_ramp=(300.0, 310.0),
                       ramp_turns=1000, t_start=-200e-9, npts=2001, lattice=LATTICE) -> str:
    """A spiral RF gap in the reference's file layout (FFAG_EField_spiral,
    src/FFAG_Field.py:379-463; written as examples/main_Emap.py:752-800,
    960-980 write theirs): emap.txt (header with gap_model = spiral, the gap
    crossing tables Ek_gap / r_gap / phi_gap_deg / phi_gap_unwrapped_deg and
    the map file names, then the frequency curve) and Er_coef.txt,
    Ez_coef.txt, Ephi_coef.txt ((nr + 1) x (nphi + 1): phi axis in the first
    row, r axis in the first column).  The gap follows the logarithmic spiral
    phi_s(r) = s_ref + tan(alpha) ln(r / r_ref); its field has a Gaussian
    profile of width sigma across the line, Eh = gap_width / (sigma
    sqrt(2 pi)) exp(-d^2 / 2 sigma^2) with d = r (phi - phi_s(r)) cos(alpha)
    (so V0 / gap_width * Eh integrates to V0 across the gap), directed along
    the line's normal (Er, Ephi) = Eh (-sin alpha, cos alpha); Ez / z =
    -(Er / r + dEr/dr + dEphi/dphi / r) by central differences.  Returns the
    emap.txt path."""
    os.makedirs(folder, exist_ok=True)
    al = math.radians(alpha_deg)
    s_ref = math.radians(s_ref_deg)
    r = np.linspace(r_axis[0], r_axis[1], int(r_axis[2]))

    def phi_s(rr):
        return s_ref + math.tan(al) * np.log(np.asarray(rr, np.float64) / r_ref)
    pad = math.radians(pad_deg)
    phi = np.linspace(float(phi_s(r).min()) - pad, float(phi_s(r).max()) + pad, int(nphi))
    R, PHI = np.meshgrid(r, phi, indexing="ij")
    d = R * (PHI - phi_s(R)) * math.cos(al)
    Eh = gap_width / (sigma * math.sqrt(2 * math.pi)) * np.exp(-0.5 * (d / sigma) ** 2)
    Er, Ephi = -math.sin(al) * Eh, math.cos(al) * Eh
    Ezc = -(Er / R + np.gradient(Er, r, axis=0) + np.gradient(Ephi, phi, axis=1) / R)
    names = {"Er_map_file": "Er_coef.txt", "Ez_map_file": "Ez_coef.txt", "Ephi_map_file": "Ephi_coef.txt"}
    for key, data in (("Er_map_file", Er), ("Ez_map_file", Ezc), ("Ephi_map_file", Ephi)):
        table = np.zeros((len(r) + 1, len(phi) + 1))
        table[0, 1:] = phi
        table[1:, 0] = r
        table[1:, 1:] = data
        np.savetxt(os.path.join(folder, names[key]), table, fmt="%.17e")
    Ek_gap = np.linspace(Ek_ramp[0] - 50.0, Ek_ramp[1] + 50.0, 11)
    r_gap = orbit_radius(Ek_gap, lattice)
    phi_gap_unwrapped = np.degrees(math.radians(gap_azimuth_deg[0]) + phi_s(r_gap))
    T0 = float(revolution_time(Ek_ramp[0], lattice))
    t = np.linspace(t_start, t_start + ramp_turns * T0 * 1.05, npts)
    frac = np.clip(t / (ramp_turns * T0), 0.0, 1.0)
    Ek = Ek_ramp[0] + (Ek_ramp[1] - Ek_ramp[0]) * frac
    f = harmonic / revolution_time(Ek, lattice)
    header = [
        "gap_model = spiral",
        f"Ngap = {len(gap_azimuth_deg)}",
        f"acc_phi_paint = {float(acc_phi_deg)}",
        f"acc_phi_acc = {float(acc_phi_deg)}",
        f"gap_azimuth = {[float(a) for a in gap_azimuth_deg]}",
        f"rf_shift = {[float(a) for a in rf_shift_deg]}",
        f"gap_width = {float(gap_width)}",
        f"harmonic = {int(harmonic)}",
        f"Ek_gap = {[float(x) for x in Ek_gap]}",
        f"r_gap = {[float(x) for x in r_gap]}",
        f"phi_gap_deg = {[float(x % 360.0) for x in phi_gap_unwrapped]}",
        f"phi_gap_unwrapped_deg = {[float(x) for x in phi_gap_unwrapped]}",
        f"dt_uniform = {float(t[1] - t[0]):.6e}",
    ] + [f"{k} = {v}" for k, v in names.items()] + ["#Time (s)        Frequency (Hz)    V0 (V)    Energy (MeV)"]
    path = os.path.join(folder, "emap.txt")
    with open(path, "w") as fh:
        fh.write("\n".join(header) + "\n")
        np.savetxt(fh, np.column_stack([t, f, np.full_like(t, voltage), Ek]), fmt="%.12e", delimiter="\t")
    return path


def seo_tables(Ek_axis=None, nfi=361, lattice=LATTICE):
    """Closed-orbit tables r0(Ek, fi), pr0(Ek, fi) and perimeter(Ek) from the
    scaling law (pr0 = 0; fi axis over [0, 2 pi])."""
    if Ek_axis is None:
        Ek_axis = np.linspace(250.0, 350.0, 101)
    fi_axis = np.linspace(0.0, 2 * np.pi, nfi)
    r0 = np.repeat(orbit_radius(Ek_axis, lattice)[:, None], nfi, axis=1)
    pr0 = np.zeros_like(r0)
    perimeter = 2 * np.pi * orbit_radius(Ek_axis, lattice)
    return {"Ek_axis": np.asarray(Ek_axis, np.float64), "fi_axis": fi_axis, "r": r0, "pr": pr0,
            "perimeter": perimeter}


def gaussian_bunch(n, seed=0, Ek=300.0, sig_x=2e-3, sig_xp=1e-3, sig_z=2e-3, sig_zp=1e-3, sig_delta=1e-3,
                   r0=None, fi0=0.0, inj_t=0.0, sig_t=0.0, lattice=LATTICE):
    """6D Gaussian bunch in p-format, sorted by inj_t, Global_ID = index."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if r0 is None:
        r0 = float(orbit_radius(Ek, lattice))
    a = np.zeros((n, 16))
    a[:, 0] = r0 + sig_x * rng.standard_normal(n)
    a[:, 1] = sig_xp * rng.standard_normal(n)
    a[:, 2] = sig_z * rng.standard_normal(n)
    a[:, 3] = sig_zp * rng.standard_normal(n)
    p0 = momentum(Ek)
    p = p0 * (1 + sig_delta * rng.standard_normal(n))
    a[:, 5] = (np.sqrt((p * C_LIGHT) ** 2 + E0_J ** 2) - E0_J) / (1e6 * Q)
    dt_ns = sig_t * 1e9 * rng.standard_normal(n) if sig_t > 0 else np.zeros(n)
    T0 = float(revolution_time(Ek, lattice))
    a[:, 4] = fi0 - 2 * np.pi * (dt_ns * 1e-9) / T0
    a[:, 6] = inj_t
    a[:, 15] = np.arange(n)
    return a


def kv_bunch(n, seed=0, Ek=300.0, a_x=4e-3, a_z=4e-3, a_xp=2e-3, a_zp=2e-3, sig_t=20e-9, fi0=np.pi,
             sig_delta=0.0, r0=None, lattice=LATTICE):
    """Transverse KV (uniform on the 4D ellipsoid surface; the x-z projection
    is a uniform ellipse) with a Gaussian longitudinal spread of sigma_t in
    time, all particles injected at t = 0 (p-format)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((n, 4))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    if r0 is None:
        r0 = float(orbit_radius(Ek, lattice))
    a = np.zeros((n, 16))
    a[:, 0] = r0 + a_x * g[:, 0]
    a[:, 1] = a_xp * g[:, 1]
    a[:, 2] = a_z * g[:, 2]
    a[:, 3] = a_zp * g[:, 3]
    p0 = momentum(Ek)
    p = p0 * (1 + sig_delta * rng.standard_normal(n)) if sig_delta > 0 else np.full(n, p0)
    a[:, 5] = (np.sqrt((p * C_LIGHT) ** 2 + E0_J ** 2) - E0_J) / (1e6 * Q)
    T0 = float(revolution_time(Ek, lattice))
    a[:, 4] = fi0 - 2 * np.pi * (sig_t * rng.standard_normal(n)) / T0
    a[:, 15] = np.arange(n)
    return a


def steps_per_turn_dt(Ek=300.0, steps_per_turn=720, lattice=LATTICE):
    return float(revolution_time(Ek, lattice)) / steps_per_turn


_design_cache = {}


def design(Ek=300.0, cfg=None):
    """Closed orbit at fi = 0 (r0 [m], pr0 = p_r/p_theta), tunes, orbit length
    and revolution time at energy Ek for the lattice `cfg` (default lattice)."""
    from . import orbit
    cfg = cfg if cfg is not None else lattice_bmap()
    key = (json.dumps(cfg, sort_keys=True), float(Ek))
    if key not in _design_cache:
        t = orbit.seo_tables(cfg, np.array([float(Ek)]), nfi=3)
        co = orbit.closed_orbits(cfg, float(Ek))
        L = float(t["perimeter"][0])
        _design_cache[key] = {"r0": float(co["r0"][0]), "pr0": float(co["pr0"][0]), "Qx": float(co["Qx"][0]),
                              "Qz": float(co["Qz"][0]), "perimeter": L,
                              "T_rev": L / float(beta_of(Ek) * C_LIGHT)}
    return _design_cache[key]


def design_dt(Ek=300.0, steps_per_turn=720, cfg=None):
    return design(Ek, cfg)["T_rev"] / steps_per_turn


def centred_bunch(n, seed=0, Ek=300.0, cfg=None, kind="gauss", **kw):
    """Bunch centred on the closed orbit (p-format pr = atan(pr0)).  A bunch
    spread in azimuth (the KV bunch's sigma_t) has every particle centred on
    the closed orbit at its own azimuth: the orbit is scalloped, so one
    radius for all would start the particles far from their local orbit
    with large radial oscillations."""
    d = design(Ek, cfg)
    if kind == "gauss":
        a = gaussian_bunch(n, seed=seed, Ek=Ek, r0=d["r0"], **kw)
    else:
        a = kv_bunch(n, seed=seed, Ek=Ek, r0=d["r0"], **kw)
    fm = np.mod(a[:, 4], 2 * np.pi)
    if np.any(fm != 0.0):
        from . import orbit
        key = ("orbit_table", json.dumps(cfg if cfg is not None else lattice_bmap(), sort_keys=True), float(Ek))
        if key not in _design_cache:
            t = orbit.seo_tables(cfg if cfg is not None else lattice_bmap(), np.array([float(Ek)]), nfi=721)
            _design_cache[key] = (t["fi_axis"], t["r"][0], t["pr"][0])
        fi_axis, r_co, pr_co = _design_cache[key]
        a[:, 0] += np.interp(fm, fi_axis, r_co) - d["r0"]
        a[:, 1] += np.arctan(np.interp(fm, fi_axis, pr_co))
    else:
        a[:, 1] += np.arctan(d["pr0"])
    return a
