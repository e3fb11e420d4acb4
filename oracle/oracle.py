"""ctypes front end of the CPU oracle (oracle/ffa_oracle.c, ffa_oracle_sc.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, used by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline legs.  It takes the same
host-side parameter objects as the product (the field / RF objects of
pyffa_b200.fields) and works on the reference's N x 16 matrix in place.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libffa_oracle.so")
LIB_FMA = os.path.join(HERE, "libffa_oracle_fma.so")
MAXG, MAXSEG, MAXPOLY, MAXHARM = 8, 16, 16, 16


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("ffa_oracle.c", "ffa_oracle_sc.c", "Makefile")]
    if force or not all(os.path.exists(x) for x in (LIB, LIB_FMA)) or \
            any(os.path.getmtime(s) > min(os.path.getmtime(LIB), os.path.getmtime(LIB_FMA)) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "all"], check=True)
    return LIB


class OrcField(C.Structure):
    _fields_ = [("nsectors", C.c_int32), ("n_spoly", C.c_int32), ("n_spolyp", C.c_int32),
                ("n_convex", C.c_int32), ("max_order", C.c_int32), ("pad0", C.c_int32),
                ("B0", C.c_double), ("k", C.c_double),
                ("spoly", C.c_double * MAXPOLY), ("spolyp", C.c_double * MAXPOLY),
                ("convex", C.c_double * (MAXSEG * 5)),
                ("r_min", C.c_double), ("r_step", C.c_double), ("r_size", C.c_int64),
                ("fi_min", C.c_double), ("fi_step", C.c_double), ("fi_size", C.c_int64),
                ("bz_stack", C.c_void_p), ("bfi_stack", C.c_void_p), ("br_stack", C.c_void_p),
                ("n_harm", C.c_int32), ("pad1", C.c_int32),
                ("harm_m", C.c_double * MAXHARM), ("harm_amp", C.c_double * MAXHARM),
                ("harm_ph", C.c_double * MAXHARM), ("harm_rmin", C.c_double * MAXHARM),
                ("harm_rmax", C.c_double * MAXHARM)]


class OrcEmap(C.Structure):
    _fields_ = [("enable", C.c_int32), ("ngaps", C.c_int32), ("physical_sum", C.c_int32), ("pad0", C.c_int32),
                ("poly_x", (C.c_double * 4) * MAXG), ("poly_y", (C.c_double * 4) * MAXG),
                ("box", (C.c_double * 4) * MAXG), ("theta_n", C.c_double * MAXG),
                ("rf_shift", C.c_double * MAXG), ("acc_Etot_uniform", C.c_double),
                ("fc_x0", C.c_double), ("fc_dx", C.c_double), ("fc_n", C.c_int64),
                ("fc_freq", C.c_void_p), ("fc_volt", C.c_void_p),
                ("er_map", C.c_void_p), ("ezc_map", C.c_void_p), ("ephi_map", C.c_void_p),
                ("nr", C.c_int64), ("nphi", C.c_int64), ("r0", C.c_double), ("dr", C.c_double),
                ("phi0", C.c_double), ("dphi", C.c_double), ("gap_az", C.c_double * MAXG)]


class OrcAperture(C.Structure):
    _fields_ = [("enable", C.c_int32), ("pad0", C.c_int32), ("rmin", C.c_double), ("rmax", C.c_double),
                ("zmin", C.c_double), ("zmax", C.c_double)]


class OrcConsts(C.Structure):
    _fields_ = [("q", C.c_double), ("c", C.c_double), ("m0", C.c_double), ("E0", C.c_double)]


class OrcSCParams(C.Structure):
    _fields_ = [("ns", C.c_int32), ("nx", C.c_int32), ("nz", C.c_int32), ("boris", C.c_int32),
                ("hockney", C.c_int32), ("pad0", C.c_int32), ("sigma_ratio", C.c_double),
                ("q_macro", C.c_double), ("speed_c", C.c_double), ("E0_rest_MeV", C.c_double),
                ("nE", C.c_int64), ("nfi", C.c_int64), ("seo_Ek", C.c_void_p), ("seo_fi", C.c_void_p),
                ("seo_r", C.c_void_p), ("seo_pr", C.c_void_p), ("seo_perimeter", C.c_void_p)]


class OrcSCDiag(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("fi_s", "fi_e", "slice_step", "mean_gamma_m1", "mean_x", "mean_z",
                                          "sigma_x", "sigma_z", "xmin", "xmax", "zmin", "zmax", "dx", "dz",
                                          "bunch_length", "q_density")] + [("count", C.c_int64)]


_lib = None
_lib_fma = None


def _bind(path):
    L = C.CDLL(path)
    L.orc_boris_step.argtypes = [C.c_double, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]
    L.orc_rk4_step.argtypes = [C.c_double, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_track.argtypes = [C.c_int, C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_int64, C.c_void_p,
                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_track.restype = C.c_double
    L.orc_track_noisy.argtypes = L.orc_track.argtypes + [C.c_uint64, C.c_int64]
    L.orc_track_noisy.restype = C.c_double
    L.orc_inject.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_void_p]
    L.orc_theta_track.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_double,
                                  C.c_double, C.c_void_p, C.c_void_p, C.c_int]
    L.orc_sc_step.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_sc_step.restype = C.c_int
    L.orc_spiral_lookup.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                    C.c_void_p, C.c_void_p]
    L.orc_spiral_lookup.restype = C.c_int
    L.orc_num_threads.restype = C.c_int
    L.orc_set_num_threads.argtypes = [C.c_int]
    return L


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = _bind(LIB)
    return _lib


def lib_fma():
    """The same oracle built with fused multiply-adds (a second, differently
    rounded float64 build; see oracle/Makefile)."""
    global _lib_fma
    if _lib_fma is None:
        build()
        _lib_fma = _bind(LIB_FMA)
    return _lib_fma


def _orc_field(bmap, keep):
    """OrcField of the product's FFAG_Bfield_analytical; arrays it points to
    are appended to `keep`."""
    f = OrcField()
    f.nsectors = int(bmap.Nsectors)
    sp = np.asarray(bmap.s_rad_polynomial, np.float64)
    spp = np.asarray(bmap.s_rad_polynomial_prime, np.float64)
    f.n_spoly, f.n_spolyp = len(sp), len(spp)
    f.spoly[:len(sp)] = sp.tolist()
    f.spolyp[:len(spp)] = spp.tolist()
    cp = np.asarray(bmap.convex_params, np.float64)
    f.n_convex = len(cp)
    f.convex[:cp.size] = cp.reshape(-1).tolist()
    f.max_order = int(bmap.max_order)
    f.B0, f.k = float(bmap.B0), float(bmap.k_value)
    f.r_min, f.r_step, f.r_size = float(bmap.r_min), float(bmap.r_step), int(bmap.r_size)
    f.fi_min, f.fi_step, f.fi_size = float(bmap.fi_min), float(bmap.fi_step), int(bmap.fi_size)
    if f.max_order >= 1:
        for name, arr in (("bz_stack", bmap.Bz_stack), ("bfi_stack", bmap.Bfi_stack), ("br_stack", bmap.Br_stack)):
            a = np.ascontiguousarray(arr, dtype=np.float64)
            keep.append(a)
            setattr(f, name, a.ctypes.data)
    return f


class ThetaTracker:
    """Azimuth-domain closed-orbit tracks (orc_theta_track), same interface
    as pyffa_b200.seo.ThetaTracker."""

    def __init__(self, bmap, q):
        self._keep = []
        self.field = _orc_field(bmap, self._keep)
        self.q = float(q)

    def run(self, x0, t_end, h, time_mode=0, traj=False, traj_cols=2):
        x0 = np.ascontiguousarray(x0, dtype=np.float64).reshape(-1, 5)
        m = x0.shape[0]
        n = int((t_end - 0) / h)
        t_points = np.linspace(0, t_end, n)
        x1 = np.zeros((m, 4))
        tr = np.zeros((m, n, traj_cols)) if traj else None
        lib().orc_theta_track(C.byref(self.field), x0.ctypes.data, m, n, int(time_mode), float(t_end), self.q,
                              x1.ctypes.data, tr.ctypes.data if traj else None, traj_cols)
        return x1, tr, t_points


class Setup:
    """Oracle parameter blocks built from the product's host-side objects
    (FFAG_Bfield_analytical, FFAG_EField_new or FFAG_EField_spiral,
    FFAG_GlobalParameters)."""

    def __init__(self, bmap, emap, gp):
        self._keep = []
        self.field = _orc_field(bmap, self._keep)
        bh = getattr(gp, "BHarmonics", None)
        if bh is not None and bh.enable_flag and bh.Nharm > 0:
            if bh.Nharm > MAXHARM:
                raise ValueError(f"at most {MAXHARM} field-error harmonics")
            self.field.n_harm = bh.Nharm
            for k in range(bh.Nharm):
                self.field.harm_m[k] = float(bh.m_arr[k])
                self.field.harm_amp[k] = float(bh.amp_arr[k])
                self.field.harm_ph[k] = float(bh.phase_arr[k])
                self.field.harm_rmin[k] = float(bh.rmin_arr[k])
                self.field.harm_rmax[k] = float(bh.rmax_arr[k])
        e = OrcEmap()
        e.enable = 1 if emap.EnableFlag else 0
        e.ngaps = len(emap.gap_azimuths)
        e.physical_sum = 1 if getattr(emap, "physical_sum", False) else 0
        if getattr(emap, "GapType", "fixed") == "spiral":
            maps = [np.ascontiguousarray(m, dtype=np.float64) for m in (emap.Er_map, emap.Ezcoef_map, emap.Ephi_map)]
            self._keep += maps
            e.er_map, e.ezc_map, e.ephi_map = (m.ctypes.data for m in maps)
            e.nr, e.nphi = int(emap.nr), int(emap.nphi)
            e.r0, e.dr, e.phi0, e.dphi = float(emap.r0), float(emap.dr), float(emap.phi0), float(emap.dphi)
            for g, az in enumerate(emap.gap_azimuths):
                e.gap_az[g] = float(az)
                e.rf_shift[g] = float(emap.rf_shift[g]) if g < len(emap.rf_shift) else 0.0
        else:
            for g, (region, theta, box) in enumerate(zip(emap.acc_regions, emap.gap_azimuths, emap.box_bounds)):
                for j in range(4):
                    e.poly_x[g][j] = float(region[j, 0])
                    e.poly_y[g][j] = float(region[j, 1])
                    e.box[g][j] = float(box[j])
                e.theta_n[g] = float(theta + np.pi / 2.0)
                e.rf_shift[g] = float(emap.rf_shift[g]) if g < len(emap.rf_shift) else 0.0
        e.acc_Etot_uniform = float(emap.acc_Etot_uniform)
        fc = emap.freq_curve
        e.fc_x0 = float(fc[0, 0])
        e.fc_dx = float(fc[1, 0] - fc[0, 0])
        e.fc_n = int(fc.shape[0])
        fr = np.ascontiguousarray(fc[:, 1])
        vo = np.ascontiguousarray(fc[:, 2])
        self._keep += [fr, vo]
        e.fc_freq, e.fc_volt = fr.ctypes.data, vo.ctypes.data
        self.emap = e
        a = OrcAperture()
        if getattr(gp, "Aperture_enable", False) and gp.Aperture_m is not None:
            a.enable = 1
            a.rmin, a.rmax, a.zmin, a.zmax = (float(x) for x in gp.Aperture_m)
        self.ap = a
        c = OrcConsts()
        c.q, c.c, c.m0, c.E0 = float(gp.q), float(gp.c), float(gp.m0), float(gp.E0)
        self.cs = c


def _mat(mat):
    if not (isinstance(mat, np.ndarray) and mat.dtype == np.float64 and mat.flags.c_contiguous and mat.shape[1] == 16):
        raise ValueError("oracle works in place on a C-contiguous float64 N x 16 matrix")
    return mat


def boris_step(setup: Setup, mat, t, dt):
    _mat(mat)
    lib().orc_boris_step(t, mat.ctypes.data, mat.shape[0], dt, C.byref(setup.field), C.byref(setup.emap),
                         C.byref(setup.ap), C.byref(setup.cs))


def rk4_step(setup: Setup, mat, t, dt):
    _mat(mat)
    lib().orc_rk4_step(t, mat.ctypes.data, mat.shape[0], dt, C.byref(setup.field), C.byref(setup.emap),
                       C.byref(setup.cs))


def track(setup: Setup, solver, mat, t_start, dt, nsteps, head=0, fused=False, noise=None):
    """Injection + push loop without space charge; returns (t_end, head).
    fused: run the build with fused multiply-adds (lib_fma).  noise: (seed,
    first step) -- flip or keep the last bit of every state value after every
    step (orc_track_noisy), a model of per-step rounding differences."""
    _mat(mat)
    h = C.c_int64(head)
    L = lib_fma() if fused else lib()
    args = (1 if solver == "Boris" else 0, mat.ctypes.data, mat.shape[0], t_start, dt, nsteps,
            C.byref(h), C.byref(setup.field), C.byref(setup.emap), C.byref(setup.ap), C.byref(setup.cs))
    if noise is None:
        t = L.orc_track(*args)
    else:
        t = L.orc_track_noisy(*args, int(noise[0]), int(noise[1]))
    return t, h.value


def spiral_lookup(setup: Setup, rf_amp, r, fi, z):
    """Spiral-gap field without the RF factor at points (r, fi, z): Er, Ez,
    Efi and the hit gap (-1: none), as the reference's Interpolation2D_EMap
    of FFAG_EField_spiral returns them (orc_spiral_lookup)."""
    r, fi, z = (np.asarray(x, np.float64).ravel() for x in (r, fi, z))
    out = np.zeros((len(r), 3))
    hit = np.zeros(len(r), np.int32)
    er, ez, ef = C.c_double(), C.c_double(), C.c_double()
    for k in range(len(r)):
        hit[k] = lib().orc_spiral_lookup(C.byref(setup.emap), float(rf_amp), r[k], fi[k], z[k], C.byref(er),
                                         C.byref(ez), C.byref(ef))
        out[k] = er.value, ez.value, ef.value
    return out[:, 0], out[:, 1], out[:, 2], hit


def detect_azimuth_crossing(pre_fi, post_fi, survive, target):
    """Restatement of detect_azimuth_crossing (src/FFAG_MathTools.py:1633-1695)
    with the mod-2-pi reduction of fast_mod_parallel (src/FFAG_MathTools.py:
    1554-1557).  Returns (crossed mask, interpolation ratio; 0 where the span
    is below 1e-12 or nothing crossed)."""
    tw = 2 * np.pi
    target = target % tw
    pre_fi = np.asarray(pre_fi, dtype=np.float64)
    post_fi = np.asarray(post_fi, dtype=np.float64)
    a = pre_fi - tw * np.floor(pre_fi / tw)
    b = post_fi - tw * np.floor(post_fi / tw)
    alive = np.asarray(survive) == 1
    fwd = b >= a
    hit_a = alive & fwd & (a <= target) & (target <= b)
    hit_b = alive & ~fwd & (((target >= a) & (target < tw)) | ((target >= 0) & (target <= b)))
    ratio = np.zeros(a.shape)
    with np.errstate(divide="ignore", invalid="ignore"):
        span_a = b - a
        ok = hit_a & (span_a > 1e-12)
        ratio[ok] = (target - a[ok]) / span_a[ok]
        span_b = (b + tw) - a
        tu = np.where(target <= b, target + tw, target)
        ok = hit_b & (span_b > 1e-12)
        ratio[ok] = (tu[ok] - a[ok]) / span_b[ok]
    return hit_a | hit_b, ratio


def track_crossings(setup: Setup, solver, mat, t_start, dt, nsteps, targets, head=0):
    """Injection + push loop that also records, step by step, the azimuth
    crossings of the reference's PositionDumpBunch (src/FFAG_dump.py:
    1098-1130, with the pre-step survival flag of UpdataPreStepNjit,
    src/FFAG_MathTools.py:2179-2201) as records of 23 values: target index,
    particle, step, ratio, pre-step r vr z vz fi f5 RF phase, the same
    post-step, post-step survival and injection flags, post-step Esc r z fi.
    Returns (records, t_end, head)."""
    _mat(mat)
    h = C.c_int64(head)
    t = t_start
    recs = []
    cols = [0, 1, 2, 3, 4, 5, 9]
    for s in range(nsteps):
        lib().orc_inject(mat.ctypes.data, mat.shape[0], t, dt, C.byref(h))
        pre = mat[:, cols].copy()
        surv = mat[:, 8].copy()
        (boris_step if solver == "Boris" else rk4_step)(setup, mat, t, dt)
        t = t + dt
        for k, tg in enumerate(targets):
            hit, ratio = detect_azimuth_crossing(pre[:, 4], mat[:, 4], surv, tg)
            idx = np.nonzero(hit)[0]
            if idx.size:
                r = np.empty((idx.size, 23))
                r[:, 0], r[:, 1], r[:, 2], r[:, 3] = k, idx, s, ratio[idx]
                r[:, 4:11] = pre[idx]
                r[:, 11:18] = mat[idx][:, cols]
                r[:, 18], r[:, 19] = mat[idx, 8], mat[idx, 7]
                r[:, 20:23] = mat[idx, 10:13]
                recs.append(r)
    out = np.vstack(recs) if recs else np.zeros((0, 23))
    return out, t, h.value


def sc_step(mat, alive, seo, ns, nx, nz, sigma_ratio, q_macro, boris=True, hockney=False,
            speed_c=2.99792458e8, E0_rest_MeV=938.2723):
    """One space-charge update in place; returns a dict of cubes, indices and
    diagnostics."""
    _mat(mat)
    N = mat.shape[0]
    p = OrcSCParams()
    p.ns, p.nx, p.nz, p.boris, p.hockney = ns, nx, nz, 1 if boris else 0, 1 if hockney else 0
    p.sigma_ratio, p.q_macro, p.speed_c, p.E0_rest_MeV = sigma_ratio, q_macro, speed_c, E0_rest_MeV
    keep = {k: np.ascontiguousarray(seo[k], dtype=np.float64) for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}
    p.nE, p.nfi = len(keep["Ek_axis"]), len(keep["fi_axis"])
    p.seo_Ek, p.seo_fi = keep["Ek_axis"].ctypes.data, keep["fi_axis"].ctypes.data
    p.seo_r, p.seo_pr, p.seo_perimeter = keep["r"].ctypes.data, keep["pr"].ctypes.data, keep["perimeter"].ctypes.data
    al = np.ascontiguousarray(alive, dtype=np.uint8)
    rho = np.zeros((ns, nz, nx), np.float32)
    phi = np.zeros((ns, nz, nx), np.float32)
    ex = np.zeros((ns, nz, nx), np.float32)
    ez = np.zeros((ns, nz, nx), np.float32)
    sidx = np.zeros(N, np.int32)
    cidx = np.zeros(N, np.int64)
    dg = OrcSCDiag()
    rc = lib().orc_sc_step(mat.ctypes.data, N, al.ctypes.data, C.byref(p), rho.ctypes.data, phi.ctypes.data,
                           ex.ctypes.data, ez.ctypes.data, sidx.ctypes.data, cidx.ctypes.data, C.byref(dg))
    diag = {n: getattr(dg, n) for n, _ in OrcSCDiag._fields_}
    return {"rc": rc, "rho": rho, "phi": phi, "ex": ex, "ez": ez, "slice_idx": sidx, "cell_idx": cidx, "diag": diag}


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())
