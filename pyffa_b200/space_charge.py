"""2.5D slice-by-slice space charge (host side).

SpaceCharge owns an ffa_sc_plan (device scratch) for one bunch and runs one
update of FFAG_Bunch.Build_2_5D_SliceGrid_sbs (src/FFAG_Bunch.py:1157-1352)
entirely on the device: the gathered fields land in the bunch's Esc columns
and, when rolled, in the two extrapolation endpoints the push kernels read
(src/FFAG_track.py:341-478).

Boundary: "periodic" reproduces the reference's solve (1/(eps0 k^2) on the
un-doubled grid, src/FFAG_SC_new.py:731-760); "hockney" is the open-boundary
solve on the doubled grid with the free-space Green's function built in
float64 for each update.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .constants import C_LIGHT, E0_J, E0_MEV, Q


def seo_from_bunch(bunch):
    """Closed-orbit tables attached to a bunch the way main_track does
    (examples/main_track.py:333-337)."""
    return {"Ek_axis": np.asarray(bunch.SEO_Ek_axis, np.float64), "fi_axis": np.asarray(bunch.SEO_fi_axis, np.float64),
            "r": np.asarray(bunch.SEO_r_matrix, np.float64), "pr": np.asarray(bunch.SEO_pr_matrix, np.float64),
            "perimeter": np.asarray(bunch.SEO_perimeter, np.float64)}


class SpaceCharge:
    def __init__(self, bunch, hockney: bool = False, seo=None):
        import torch
        self.bunch = bunch
        self.hockney = bool(hockney)
        seo = seo if seo is not None else seo_from_bunch(bunch)
        dev = bunch.device
        self._seo = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in seo.items()}
        Ek, fi = seo["Ek_axis"], seo["fi_axis"]
        if seo["r"].shape != (len(Ek), len(fi)) or seo["pr"].shape != (len(Ek), len(fi)):
            raise ValueError("closed-orbit tables must have shape (len(Ek_axis), len(fi_axis))")
        d = _lib.SCDesc()
        d.ns, d.nx, d.nz = bunch.f_grid_size, bunch.x_grid_size, bunch.z_grid_size
        d.hockney = 1 if self.hockney else 0
        d.boris = 1 if bunch.BunchType == "Boris" else 0
        d.n_max = bunch.n
        d.sigma_ratio = float(bunch.sigma_ratio)
        d.q_macro = float(bunch.marcosize * bunch.q_charge)
        d.speed_c, d.E0_rest_MeV, d.E0_J = C_LIGHT, E0_MEV, E0_J
        d.nE, d.nfi = len(Ek), len(fi)
        d.Ek0, d.dEk = float(Ek[0]), float(Ek[1] - Ek[0])
        d.fi0, d.dfi = float(fi[0]), float(fi[1] - fi[0])
        d.seo_Ek = self._seo["Ek_axis"].data_ptr()
        d.seo_r = self._seo["r"].data_ptr()
        d.seo_pr = self._seo["pr"].data_ptr()
        d.seo_perimeter = self._seo["perimeter"].data_ptr()
        self.desc = d
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ffa_sc_plan_create(ctypes.byref(d), _lib.stream_ptr(None), ctypes.byref(h)),
                   "ffa_sc_plan_create")
        self.handle = h
        self.diag_dev = torch.zeros(ctypes.sizeof(_lib.SCDiag) // 8, dtype=torch.float64, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def __del__(self):
        try:
            if self.handle:
                _lib.lib().ffa_sc_plan_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def update(self, first: bool = False, roll: bool = True) -> None:
        b = self.bunch
        _lib.check(_lib.lib().ffa_sc_step(self.handle, ctypes.byref(b.soa()), b.n, 1 if roll else 0,
                                          1 if first else 0, self.stream.cuda_stream, b.status.data_ptr(),
                                          self.diag_dev.data_ptr()), "ffa_sc_step")

    def diag(self) -> dict:
        raw = self.diag_dev.cpu().numpy().tobytes()
        dg = _lib.SCDiag.from_buffer_copy(raw)
        return {name: getattr(dg, name) for name, _ in _lib.SCDiag._fields_}

    def buffers(self) -> dict:
        """Copies of the last update's cubes (ns, nz, nx) and per-particle indices."""
        import torch
        L = _lib.lib()
        ptrs = [ctypes.c_void_p() for _ in range(6)]
        _lib.check(L.ffa_sc_buffers(self.handle, *[ctypes.byref(p) for p in ptrs]), "ffa_sc_buffers")
        d = self.desc
        shape = (d.ns, d.nz, d.nx)
        cube = int(np.prod(shape))
        n = self.bunch.n
        torch.cuda.synchronize(self.bunch.device)
        out = {}
        for name, p, count, ctype, dt in (("rho", ptrs[0], cube, ctypes.c_float, np.float32),
                                          ("phi", ptrs[1], cube, ctypes.c_float, np.float32),
                                          ("ex", ptrs[2], cube, ctypes.c_float, np.float32),
                                          ("ez", ptrs[3], cube, ctypes.c_float, np.float32),
                                          ("slice_idx", ptrs[4], n, ctypes.c_int32, np.int32),
                                          ("cell_idx", ptrs[5], n, ctypes.c_int64, np.int64)):
            host = np.empty(count, dtype=dt)
            _cuda_memcpy_d2h(host, p.value, host.nbytes)
            out[name] = host.reshape(shape) if count == cube and name not in ("slice_idx", "cell_idx") else host
        return out


_cudart = None


def _cuda_memcpy_d2h(host: np.ndarray, dev_ptr: int, nbytes: int) -> None:
    """Device -> host copy of a raw device pointer through torch (no extra deps)."""
    import torch
    if nbytes == 0:
        return
    # wrap the device memory as a byte tensor via the CUDA array interface
    class _Wrap:
        def __init__(self, ptr, n):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}
    t = torch.as_tensor(_Wrap(dev_ptr, nbytes), device="cuda")
    host_bytes = host.view(np.uint8).reshape(-1)
    host_bytes[:] = t.cpu().numpy()
