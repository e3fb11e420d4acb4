"""Field models of the tracking path: the scaling-FFAG mid-plane map with its
z-Taylor tables, the fixed RF gaps with their frequency curve, and the
field-error harmonics switch.

Host side of FFAG_Bfield_analytical (src/FFAG_Field.py:635-944),
FFAG_EField_new (src/FFAG_Field.py:167-376) and FFAG_BField_Error
(src/FFAG_Field.py:947-1042).  The per-particle evaluation runs in the CUDA
push kernels; this module prepares the parameters exactly as the reference
does (same axis rules, same polynomial fit, same gap geometry), since any
difference here is a difference in the physics inputs.
"""
from __future__ import annotations

import ast
import json
import os

import numpy as np

from . import _lib


# ------------------------------------------------------------------ B field

def calculate_s(r_axis, s0, alpha_deg):
    """Spiral azimuth s(r), src/FFAG_Field.py:800-823 (sequential sum)."""
    s = np.zeros_like(r_axis)
    s[0] = s0
    tan_alpha = np.tan(np.deg2rad(alpha_deg))
    for i in range(1, len(r_axis)):
        s[i] = s[i - 1] + tan_alpha / r_axis[i] * (r_axis[i] - r_axis[i - 1])
    return s


def polyder_coeffs(coeffs):
    """Derivative of a highest-degree-first polynomial (src/FFAG_Field.py:1214-1230)."""
    n = len(coeffs) - 1
    out = np.empty(n, dtype=coeffs.dtype)
    for i in range(n):
        out[i] = coeffs[i] * (n - i)
    return out


def convex_params(bmap: dict) -> np.ndarray:
    """Flutter segments (x0, x1, W0, |pol|, sign) in rad,
    BmapParams_to_ConvexParams, src/FFAG_Field.py:732-767."""
    total = 360.0 / bmap["NSector"]
    out = []
    start = 0
    for interval, pol, fringe in zip(bmap["interval_1"], bmap["positive_or_negative_1"], bmap["fringe_width_1"]):
        if pol == 0:
            start += interval * total
            continue
        end = start + interval * total
        # the reference's negative branch builds the tuple (|pol|, -1, 0)
        shape = (abs(pol), 1.0) if pol > 0 else (abs(pol), -1)
        edge = (end - start) * fringe
        out.append((np.deg2rad(start), np.deg2rad(end), np.deg2rad(edge), np.float64(shape[0]), np.float64(shape[1])))
        start = end
    return np.array(out, dtype=np.float64).reshape(-1, 5)


class FFAG_Bfield_analytical:
    """Scaling-FFAG field B0 r^k F(theta - s(r)) plus z-Taylor maps.

    Parameters follow the reference constructor (src/FFAG_Field.py:636-711):
    the JSON file's "Bmap" block and, with AddNumricalMap, the per-order
    files Br/Bz/Bfi_order_n.npz in the JSON file's folder.  ``stacks`` may be
    given directly as (Bz, Bfi, Br) arrays of shape (max_order+1, NX, NY).
    """

    def __init__(self, config_Bmap_path=None, max_order=0, flag3D=True, AddNumricalMap=True,
                 config=None, stacks=None):
        if config is None:
            with open(config_Bmap_path, "r") as f:
                config = json.load(f)
        bm = config["Bmap"]
        rmin, rmax, rstep = bm["rmin_max_step_m"]
        self.Nsectors = bm["NSector"]
        self.Bmean = bm.get("Bmean")
        theta_step = bm["theta_step_rad"]
        n_fi = int((2 * np.pi / self.Nsectors) / theta_step) + 1
        fi_axis = np.linspace(0, 2 * np.pi / self.Nsectors, n_fi)
        n_r = int((rmax - rmin) / rstep) + 1
        r_axis = np.linspace(rmin, rmax, n_r)
        s_val = calculate_s(r_axis, 0.0, bm["SpiralAngle_deg"])
        self.s_rad_polynomial = np.polyfit(r_axis, s_val, 6)
        self.s_rad_polynomial_prime = polyder_coeffs(self.s_rad_polynomial)
        self.B0, self.k_value = bm["coefficients_tupel"]
        self.r_axis, self.fi_axis = r_axis, fi_axis
        self.r_min, self.r_max, self.r_step = rmin, rmax, rstep
        self.fi_min, self.fi_max = fi_axis[0], fi_axis[-1]
        self.fi_step = fi_axis[1] - fi_axis[0]
        self.r_size, self.fi_size = len(r_axis), len(fi_axis)
        self.convex_params = convex_params(bm)
        self.r_axis_Bmean = bm.get("r_axis")
        self.f1 = None
        if self.Bmean is not None:
            from scipy.interpolate import interp1d
            self.f1 = interp1d(self.r_axis_Bmean, self.Bmean, kind="linear", fill_value="extrapolate")
        self.max_order = int(max_order)
        self.flag3D = flag3D
        self.config_path = config_Bmap_path
        self.BmapFoldName = os.path.dirname(config_Bmap_path) if config_Bmap_path else None
        self.Bz_stack = self.Bfi_stack = self.Br_stack = None
        if stacks is not None:
            self.Bz_stack, self.Bfi_stack, self.Br_stack = (np.ascontiguousarray(s, dtype=np.float64) for s in stacks)
        elif AddNumricalMap and self.max_order >= 1:
            fold = os.path.normpath(self.BmapFoldName)
            br, bz, bfi = [], [], []
            for n in range(0, self.max_order + 1):
                br.append(np.load(os.path.join(fold, f"Br_order_{n}.npz"))["Br_Taylor_coeff"])
                bz.append(np.load(os.path.join(fold, f"Bz_order_{n}.npz"))["Bz_Taylor_coeff"])
                bfi.append(np.load(os.path.join(fold, f"Bfi_order_{n}.npz"))["Bfi_Taylor_coeff"])
            self.Br_stack = np.ascontiguousarray(np.stack(br, axis=0))
            self.Bz_stack = np.ascontiguousarray(np.stack(bz, axis=0))
            self.Bfi_stack = np.ascontiguousarray(np.stack(bfi, axis=0))
        if self.max_order >= 1:
            for s in (self.Bz_stack, self.Bfi_stack, self.Br_stack):
                if s is None or s.shape[0] < self.max_order + 1 or s.shape[1:] != (self.r_size, self.fi_size):
                    raise ValueError(
                        f"z-Taylor stack must have shape (>= {self.max_order + 1}, {self.r_size}, {self.fi_size})")
        self._device = {}

    # -- host evaluation of the mid-plane field (table setup only)
    def GetBz(self, r, fi):
        """Mid-plane Bz = B0 r^k F(fi - s(r)) on the host (GetBz,
        src/FFAG_Field.py:794-815, without the search-mode clamp)."""
        r = np.asarray(r, dtype=np.float64)
        fi = np.asarray(fi, dtype=np.float64)
        s = np.zeros_like(r)
        for c in self.s_rad_polynomial:
            s = s * r + c
        amp = self.B0 * np.power(r, self.k_value)
        period = 2 * np.pi / self.Nsectors
        x = fi - s
        x = x - period * np.floor(x / period)
        F = x * 0.0
        for x0, x1, W0, y01, y02 in self.convex_params:
            k = 16 / W0
            F += y02 * np.abs(y01) * (1 / (1 + np.exp(-k * (x - x0)))) * (1 / (1 + np.exp(k * (x - x1))))
        return amp * F

    def UpdataConfig(self, save_folder=None):
        """Sector-mean field per radius, written back into the lattice JSON
        as Bmap.Bmean / Bmap.r_axis (UpdataConfig, src/FFAG_Field.py:904-943);
        the closed-orbit search starts from it (func_get_R_B0)."""
        from scipy.interpolate import interp1d
        self.Bmean = [float(np.mean(self.GetBz(np.full_like(self.fi_axis, r), self.fi_axis))) for r in self.r_axis]
        self.r_axis_Bmean = self.r_axis.tolist()
        self.f1 = interp1d(self.r_axis_Bmean, self.Bmean, kind="linear", fill_value="extrapolate")
        if self.config_path:
            with open(self.config_path) as f:
                cfg = json.load(f)
            cfg["Bmap"]["Bmean"] = self.Bmean
            cfg["Bmap"]["r_axis"] = self.r_axis_Bmean
            folder = save_folder or self.BmapFoldName
            with open(os.path.join(folder, "config_Bmap.json"), "w") as f:
                json.dump(cfg, f, indent=4)

    # -- kernel descriptor
    def field_desc(self) -> "_lib.FieldDesc":
        d = _lib.FieldDesc()
        d.nsectors = int(self.Nsectors)
        sp, spp = np.asarray(self.s_rad_polynomial, np.float64), np.asarray(self.s_rad_polynomial_prime, np.float64)
        if len(sp) > _lib.MAX_POLY or len(self.convex_params) > _lib.MAX_SEG:
            raise ValueError("spiral polynomial or flutter segment count exceeds the kernel limits")
        d.n_spoly, d.n_spolyp = len(sp), len(spp)
        d.spoly[:len(sp)] = sp.tolist()
        d.spolyp[:len(spp)] = spp.tolist()
        d.n_convex = len(self.convex_params)
        d.convex[:5 * d.n_convex] = self.convex_params.reshape(-1).tolist()
        d.max_order = self.max_order
        d.B0, d.k = float(self.B0), float(self.k_value)
        d.r_min, d.r_step, d.r_size = float(self.r_min), float(self.r_step), int(self.r_size)
        d.fi_min, d.fi_step, d.fi_size = float(self.fi_min), float(self.fi_step), int(self.fi_size)
        return d

    def device_map(self, device):
        """Packed device field map (cached per device)."""
        import torch
        key = str(device)
        if key in self._device:
            return self._device[key]
        d = self.field_desc()
        keep = []
        if self.max_order >= 1:
            n = self.max_order + 1
            for name in ("bz_stack", "bfi_stack", "br_stack"):
                src = {"bz_stack": self.Bz_stack, "bfi_stack": self.Bfi_stack, "br_stack": self.Br_stack}[name]
                t = torch.from_numpy(np.ascontiguousarray(src[:n])).to(device)
                keep.append(t)
                setattr(d, name, t.data_ptr())
        fm = DeviceFieldMap(d, device)
        torch.cuda.synchronize(device)  # the pack kernel has read the stacks
        del keep
        self._device[key] = fm
        return fm


class DeviceFieldMap:
    """Owner of an ffa_fieldmap handle."""

    def __init__(self, desc, device):
        import ctypes
        import torch
        self.desc = desc
        self.device = device
        h = ctypes.c_void_p()
        with torch.cuda.device(device):
            _lib.check(_lib.lib().ffa_fieldmap_create(ctypes.byref(desc), _lib.stream_ptr(None), ctypes.byref(h)),
                       "ffa_fieldmap_create")
        self.handle = h
        self._harm_key = ()

    def set_harmonics(self, harmonics) -> None:
        """Makes the map carry the field-error harmonics of an
        FFAG_BField_Error (None or disabled: none).  The library copies them
        to the device synchronously, so this is done only when they change."""
        import ctypes
        import torch
        if harmonics is not None and harmonics.active():
            arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                    (harmonics.m_arr, harmonics.amp_arr, harmonics.phase_arr, harmonics.rmin_arr, harmonics.rmax_arr)]
        else:
            arrs = []
        key = tuple(tuple(a.tolist()) for a in arrs)
        if key == self._harm_key:
            return
        ptrs = [ctypes.c_void_p(a.ctypes.data) for a in arrs] if arrs else [None] * 5
        with torch.cuda.device(self.device):
            _lib.check(_lib.lib().ffa_fieldmap_set_harmonics(self.handle, len(arrs[0]) if arrs else 0, *ptrs),
                       "ffa_fieldmap_set_harmonics")
        self._harm_key = key

    def __del__(self):
        try:
            if self.handle:
                _lib.lib().ffa_fieldmap_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


# ------------------------------------------------------------------ E field

def parse_emap_file(file_path):
    """Header key = value pairs and the data table of an Emap frequency-curve
    file, with the reference's value typing (ParseEmapFile,
    src/FFAG_Field.py:316-376)."""
    params = {}
    non_data = 0
    with open(file_path, "r") as f:
        for line in f:
            line = line.strip()
            if line.startswith("#Time (s)"):
                non_data += 1
                break
            if "=" in line:
                key, value = (s.strip() for s in line.split("=", 1))
                try:
                    if "." in value or "e" in value.lower():
                        params[key] = float(value)
                    else:
                        params[key] = int(value)
                except ValueError:
                    parsed = None
                    if (value.startswith("[") and value.endswith("]")) or (value.startswith("(") and value.endswith(")")):
                        try:
                            obj = ast.literal_eval(value)
                            if isinstance(obj, (list, tuple)):
                                parsed = [float(x) for x in obj]
                        except Exception:
                            parsed = None
                    if parsed is None and "," in value:
                        parts = [p.strip() for p in value.split(",") if p.strip() != ""]
                        try:
                            parsed = [float(p) if ("." in p or "e" in p.lower()) else float(int(p)) for p in parts]
                        except Exception:
                            parsed = None
                    params[key] = parsed if parsed is not None else value
            non_data += 1
    data = np.loadtxt(file_path, skiprows=non_data)
    return params, data


class FFAG_EField_new:
    """Fixed rectangular RF gaps driven by a frequency/voltage curve
    (src/FFAG_Field.py:167-376)."""

    GapType = "fixed"

    def __init__(self, freq_curve_path=None, EnableFlag=True, header=None, data=None):
        if header is None:
            header, data = parse_emap_file(freq_curve_path)
        self.header = header
        self.acc_phi0 = np.deg2rad(header["acc_phi_paint"])
        self.gap_azimuths = np.deg2rad(np.atleast_1d(header["gap_azimuth"]))
        self.gap_width = header["gap_width"]
        self.rmin = header["E_rmin"]
        self.rmax = header["E_rmax"]
        self.freq_curve = np.asarray(data, dtype=np.float64)
        self.harmonic = header["harmonic"]
        self.EnableFlag = EnableFlag
        self.rf_shift = np.deg2rad(np.atleast_1d(header["rf_shift"]))
        if len(self.gap_azimuths) > _lib.MAX_GAPS:
            raise ValueError(f"at most {_lib.MAX_GAPS} RF gaps are supported")
        self.acc_regions = self.compute_acc_region()
        self.box_bounds = []
        for region in self.acc_regions:
            self.box_bounds.append((np.min(region[:, 0]), np.max(region[:, 0]),
                                    np.min(region[:, 1]), np.max(region[:, 1])))
        self.acc_Etot_uniform = 1 / self.gap_width
        self.physical_sum = False

    def compute_acc_region(self):
        """Gap rectangles (4 x 2 vertices each), src/FFAG_Field.py:236-261."""
        regions = []
        for theta in np.atleast_1d(self.gap_azimuths):
            cs = np.array([self.rmin * np.cos(theta), self.rmin * np.sin(theta)])
            ce = np.array([self.rmax * np.cos(theta), self.rmax * np.sin(theta)])
            n = np.array([np.cos(theta + np.pi / 2), np.sin(theta + np.pi / 2)])
            regions.append(np.stack([cs + 0.5 * self.gap_width * n, ce + 0.5 * self.gap_width * n,
                                     ce - 0.5 * self.gap_width * n, cs - 0.5 * self.gap_width * n]))
        return regions

    def Interpolation1D_freq_curve(self, time):
        """(f_rf, V0) at `time`, linear_interpolation_uniform_njit_two_vars
        (src/FFAG_MathTools.py:1431-1478); vectorised over `time`."""
        X0 = self.freq_curve[0, 0]
        dX = self.freq_curve[1, 0] - self.freq_curve[0, 0]
        Y, Z = self.freq_curve[:, 1], self.freq_curve[:, 2]
        xi = np.asarray(time, dtype=np.float64)
        N = Y.shape[0]
        i = np.floor((xi - X0) / dX).astype(np.int64)
        i = np.where(i < 0, 0, np.where(i >= N - 1, N - 2, i))
        x0 = X0 + i * dX
        x1 = x0 + dX
        yi = Y[i] + (xi - x0) / (x1 - x0) * (Y[i + 1] - Y[i])
        zi = Z[i] + (xi - x0) / (x1 - x0) * (Z[i + 1] - Z[i])
        return yi, zi

    def rf_desc(self, device=None) -> "_lib.RFDesc":
        """The push kernels' description of the gaps (device: unused, the
        fixed gaps need no device table)."""
        d = _lib.RFDesc()
        d.enable = 1 if self.EnableFlag else 0
        d.ngaps = len(self.gap_azimuths)
        for g, (region, theta, box) in enumerate(zip(self.acc_regions, self.gap_azimuths, self.box_bounds)):
            for j in range(4):
                d.poly_x[g][j] = float(region[j, 0])
                d.poly_y[g][j] = float(region[j, 1])
            for j in range(4):
                d.box[g][j] = float(box[j])
            d.theta_n[g] = float(theta + np.pi / 2.0)
            d.rf_shift[g] = float(self.rf_shift[g] if g < len(self.rf_shift) else 0.0)
        return d


def load_spiral_map(path):
    """A spiral E-map file: first row the phi axis (from column 1), first
    column the r axis (from row 1), the rest the (nr, nphi) values
    (FFAG_EField_spiral.LoadSpiralMap, src/FFAG_Field.py:458-463)."""
    raw = np.loadtxt(path)
    return raw[1:, 1:].astype(np.float64), raw[1:, 0].astype(np.float64), raw[0, 1:].astype(np.float64)


class FFAG_EField_spiral:
    """Spiral RF gaps (src/FFAG_Field.py:379-550): one (r, phi) map of Er,
    Ez / z and Ephi, placed at every gap azimuth, driven by the frequency /
    voltage curve.  The push kernels evaluate it (interpolate_spiral_emap_
    unique_gap_kernel, src/FFAG_MathTools.py:1042-1114: the first gap whose
    window holds the particle, bilinear in (r, phi), E = V0 / gap_width *
    map * sin(RF phase + rf_shift)); the map goes to the device with the
    first rf_desc on a device.  Ek_gap / r_gap / phi_gap tables give the gap
    crossing of the closed orbit per energy (r_gap_interp,
    phi_gap_interp_unwrapped: linear interpolation, as np.interp)."""

    GapType = "spiral"

    def __init__(self, freq_curve_path=None, EnableFlag=True, header=None, data=None):
        if header is None:
            header, data = parse_emap_file(freq_curve_path)
        self.header = header
        self.acc_phi0 = np.deg2rad(float(header["acc_phi_paint"]))
        self.gap_azimuths = np.deg2rad(np.atleast_1d(header["gap_azimuth"]).astype(np.float64))
        if len(self.gap_azimuths) > _lib.MAX_GAPS:
            raise ValueError(f"at most {_lib.MAX_GAPS} RF gaps are supported")
        self.gap_width = float(header["gap_width"])
        self.freq_curve = np.asarray(data, dtype=np.float64)
        self.harmonic = int(header["harmonic"])
        self.EnableFlag = EnableFlag
        self.rf_shift = np.deg2rad(np.atleast_1d(header["rf_shift"]).astype(np.float64))
        folder = os.path.dirname(os.path.abspath(freq_curve_path)) if freq_curve_path else "."
        self.Er_map, self.r_axis, self.phi_axis = load_spiral_map(
            os.path.join(folder, header.get("Er_map_file", "Er_coef.txt")))
        self.Ezcoef_map = load_spiral_map(os.path.join(folder, header.get("Ez_map_file", "Ez_coef.txt")))[0]
        self.Ephi_map = load_spiral_map(os.path.join(folder, header.get("Ephi_map_file", "Ephi_coef.txt")))[0]
        if not (self.Er_map.shape == self.Ezcoef_map.shape == self.Ephi_map.shape):
            raise ValueError("the three spiral maps differ in shape")
        self.r0, self.dr, self.nr = self.r_axis[0], self.r_axis[1] - self.r_axis[0], len(self.r_axis)
        self.phi0, self.dphi, self.nphi = self.phi_axis[0], self.phi_axis[1] - self.phi_axis[0], len(self.phi_axis)
        self.map_rmin, self.map_rmax = self.r_axis[0], self.r_axis[-1]
        self.map_phimin, self.map_phimax = self.phi_axis[0], self.phi_axis[-1]
        self.acc_Etot_uniform = 1.0 / self.gap_width
        order = np.argsort(np.atleast_1d(header["Ek_gap"]).astype(np.float64))
        self.Ek_gap = np.atleast_1d(header["Ek_gap"]).astype(np.float64)[order]
        self.r_gap = np.atleast_1d(header["r_gap"]).astype(np.float64)[order]
        self.phi_gap = np.deg2rad(np.atleast_1d(header["phi_gap_deg"]).astype(np.float64))[order]
        self.phi_gap_unwrapped = np.deg2rad(np.atleast_1d(header["phi_gap_unwrapped_deg"]).astype(np.float64))[order]
        self.physical_sum = False
        self._nodes = {}

    def r_gap_interp(self, Ek):
        return np.interp(np.asarray(Ek, np.float64), self.Ek_gap, self.r_gap)

    def phi_gap_interp_unwrapped(self, Ek):
        return np.interp(np.asarray(Ek, np.float64), self.Ek_gap, self.phi_gap_unwrapped)

    Interpolation1D_freq_curve = FFAG_EField_new.Interpolation1D_freq_curve

    def device_nodes(self, device):
        """The (nr, nphi, 4) float64 node table on `device`: Er, Ez / z,
        Ephi, 0 per node (kept for the object's lifetime)."""
        import torch
        key = str(torch.device(device))
        if key not in self._nodes:
            t = np.stack([self.Er_map, self.Ezcoef_map, self.Ephi_map, np.zeros_like(self.Er_map)], axis=-1)
            self._nodes[key] = torch.as_tensor(np.ascontiguousarray(t), device=device)
        return self._nodes[key]

    def rf_desc(self, device=None) -> "_lib.RFDesc":
        """The push kernels' description of the gaps, with the node table
        on `device` (default: the current CUDA device)."""
        import torch
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        d = _lib.RFDesc()
        d.enable = 1 if self.EnableFlag else 0
        d.ngaps = len(self.gap_azimuths)
        for g, az in enumerate(self.gap_azimuths):
            d.gap_azimuth[g] = float(az)
            d.rf_shift[g] = float(self.rf_shift[g] if g < len(self.rf_shift) else 0.0)
        d.spiral_nodes = self.device_nodes(device).data_ptr()
        d.spiral_nr, d.spiral_nphi = int(self.nr), int(self.nphi)
        d.spiral_r0, d.spiral_dr = float(self.r0), float(self.dr)
        d.spiral_phi0, d.spiral_dphi = float(self.phi0), float(self.dphi)
        return d


class FFAG_BField_Error:
    """Field-error harmonics (src/FFAG_Field.py:947-993): Bz(r, fi) gains
    sum_k amp_k cos(m_k fi + phase_k) for rmin_k <= r <= rmax_k, with fi the
    unwrapped azimuth; Br and Bfi are unchanged.  `harmonics_cfg` is a list
    of dicts {"m", "amp_Gs", "phase_deg", "rmin", "rmax"} (gauss, degrees,
    metres), as in the reference.  The push kernels add the sum after the
    mid-plane map (Boris_solve src/FFAG_track.py:1007, the RK4 field
    FunctionForAccelerationBunch_dt :1782)."""

    MAX_HARMONICS = 16

    def __init__(self, harmonics_cfg, EnableFlag):
        self.harmonics_cfg = harmonics_cfg
        self.enable_flag = bool(EnableFlag)
        self.Nharm = len(harmonics_cfg)
        if self.Nharm > self.MAX_HARMONICS:
            raise ValueError(f"at most {self.MAX_HARMONICS} field-error harmonics")
        self.m_arr = np.array([int(h["m"]) for h in harmonics_cfg], dtype=np.int64)
        self.amp_arr = np.array([float(h["amp_Gs"]) * 1e-4 for h in harmonics_cfg], dtype=np.float64)
        self.phase_arr = np.array([np.deg2rad(float(h["phase_deg"])) for h in harmonics_cfg], dtype=np.float64)
        self.rmin_arr = np.array([float(h["rmin"]) for h in harmonics_cfg], dtype=np.float64)
        self.rmax_arr = np.array([float(h["rmax"]) for h in harmonics_cfg], dtype=np.float64)

    def active(self) -> bool:
        return self.enable_flag and self.Nharm > 0

    def GetBzHarmonics(self, r, phi):
        """Bz of the harmonics at (r, phi), numpy, broadcasting."""
        r = np.asarray(r, np.float64)
        phi = np.asarray(phi, np.float64)
        out = np.zeros(np.broadcast(r, phi).shape)
        if not self.enable_flag:
            return out
        for k in range(self.Nharm):
            band = (self.rmin_arr[k] <= r) & (r <= self.rmax_arr[k])
            out = out + np.where(band, self.amp_arr[k] * np.cos(self.m_arr[k] * phi + self.phase_arr[k]), 0.0)
        return out