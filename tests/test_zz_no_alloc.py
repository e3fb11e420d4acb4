"""The space-charge update that allocates nothing (ffa_sc_step_static).

Callers that cannot allocate device memory while they run (a host code
that reserves its device budget up front, or a tracking loop inside a
control system where an allocation could fail or stall the device) use
ffa_sc_step_static instead of ffa_sc_plan_create + ffa_sc_step.  This test
calls it through the C ABI and checks, on calls in a row with different
bunches and grids (128 x 128 twice, then 64 x 64, then 32 x 16, which takes
the batched-FFT path), that it gives what the plan-based update gives on the
same input: both run the same kernels on the same input, so every
result must be identical.  Around a warm call the device's free memory must not change.
It also checks that sizes beyond the fixed scratch are refused up front.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


@pytest.fixture(scope="module")
def seo():
    from pyffa_b200 import orbit, synthetic
    t = orbit.seo_tables(synthetic.lattice_bmap(), np.linspace(290.0, 310.0, 9), nfi=361)
    return {k: t[k] for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}


def _matrix(n, seed):
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    p = synthetic.centred_bunch(n, seed=seed, kind="kv", a_x=4e-3, a_z=3e-3, sig_t=20e-9, fi0=2.0)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    v[: n // 50, 8] = 0.0
    return v


def _bunch(v, grid, seo):
    from pyffa_b200.bunch import FFAG_Bunch
    b = FFAG_Bunch(v, marcosize=1e13 / v.shape[0], sc_grid_size=grid, BunchType="Boris")
    b.SEO_fi_axis, b.SEO_Ek_axis = seo["fi_axis"], seo["Ek_axis"]
    b.SEO_r_matrix, b.SEO_pr_matrix, b.SEO_perimeter = seo["r"], seo["pr"], seo["perimeter"]
    return b


def _desc(b, seo, keep, hockney=False):
    """The same descriptor SpaceCharge builds, with caller-owned table tensors."""
    from pyffa_b200 import _lib
    from pyffa_b200.constants import C_LIGHT, E0_J, E0_MEV
    for k, v in seo.items():
        keep[k] = torch.from_numpy(np.ascontiguousarray(v)).to(b.device)
    d = _lib.SCDesc()
    d.ns, d.nx, d.nz = b.f_grid_size, b.x_grid_size, b.z_grid_size
    d.hockney = 1 if hockney else 0
    d.boris = 1
    d.n_max = b.n
    d.sigma_ratio = float(b.sigma_ratio)
    d.q_macro = float(b.marcosize * b.q_charge)
    d.speed_c, d.E0_rest_MeV, d.E0_J = C_LIGHT, E0_MEV, E0_J
    d.nE, d.nfi = len(seo["Ek_axis"]), len(seo["fi_axis"])
    d.Ek0, d.dEk = float(seo["Ek_axis"][0]), float(seo["Ek_axis"][1] - seo["Ek_axis"][0])
    d.fi0, d.dfi = float(seo["fi_axis"][0]), float(seo["fi_axis"][1] - seo["fi_axis"][0])
    d.seo_Ek, d.seo_r = keep["Ek_axis"].data_ptr(), keep["r"].data_ptr()
    d.seo_pr, d.seo_perimeter = keep["pr"].data_ptr(), keep["perimeter"].data_ptr()
    return d


def _static_update(b, d, first, check_free=False):
    from pyffa_b200 import _lib
    diag = torch.zeros(ctypes.sizeof(_lib.SCDiag) // 8, dtype=torch.float64, device=b.device)
    soa = b.soa()
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = _lib.lib().ffa_sc_step_static(ctypes.byref(d), ctypes.byref(soa), b.n, 1, 1 if first else 0,
                                       stream, b.status.data_ptr(), diag.data_ptr())
    assert rc == 0
    torch.cuda.synchronize()
    if check_free:
        assert torch.cuda.mem_get_info()[0] == free0
    dg = _lib.SCDiag.from_buffer_copy(diag.cpu().numpy().tobytes())
    return {name: getattr(dg, name) for name, _ in _lib.SCDiag._fields_}


def _endpoints(b):
    return {k: b.cols[k].cpu().numpy() for k in ("e_pre_r", "e_pre_z", "e_pre_fi", "e_pp_r", "e_pp_z", "e_pp_fi",
                                                 "sc_pre", "sc_pp")}


CALLS = (((16, 128, 128, 12.0), 200_000, 1), ((16, 128, 128, 12.0), 150_000, 2),
         ((8, 64, 64, 12.0), 60_000, 4), ((8, 32, 16, 12.0), 30_000, 5))


def test_static_update_matches_plan_update(seo):
    from pyffa_b200.space_charge import SpaceCharge
    for call, (grid, n, seed) in enumerate(CALLS):
        v = _matrix(n, seed)
        a = _bunch(v, grid, seo)
        sc = SpaceCharge(a)
        sc.update(first=(call == 0), roll=True)
        ref_diag = sc.diag()

        b = _bunch(v, grid, seo)
        keep = {}
        # from the second call on the library's module is loaded: a call must
        # then leave the device's free memory as it found it
        got_diag = _static_update(b, _desc(b, seo, keep), first=(call == 0), check_free=(call > 0))

        for k in ("fi_s", "fi_e", "slice_step", "mean_gamma_m1", "xmin", "xmax", "zmin", "zmax", "dx", "dz",
                  "bunch_length", "q_density", "count", "degenerate"):
            assert got_diag[k] == ref_diag[k], (call, k)
        ma, mb = a.LocalBunch, b.LocalBunch
        for c in (10, 11, 12):
            assert np.array_equal(ma[:, c], mb[:, c]), (call, c)
        ea, eb = _endpoints(a), _endpoints(b)
        assert np.array_equal(ea["sc_pre"], eb["sc_pre"]) and np.array_equal(ea["sc_pp"], eb["sc_pp"])
        for k in ("e_pre_r", "e_pre_z", "e_pre_fi", "e_pp_r", "e_pp_z", "e_pp_fi"):
            assert np.array_equal(ea[k], eb[k]), (call, k)
        assert np.array_equal(ma[:, :10], mb[:, :10])


def test_static_update_rejects_oversize(seo):
    from pyffa_b200 import _lib
    v = _matrix(1000, 3)
    b = _bunch(v, (16, 128, 128, 12.0), seo)
    keep = {}
    d = _desc(b, seo, keep)
    L = _lib.lib()
    s = torch.cuda.current_stream().cuda_stream
    too_many = _lib.SC_STATIC_MAX_PARTICLES + 1
    assert L.ffa_sc_step_static(ctypes.byref(d), ctypes.byref(b.soa()), too_many, 0, 1, s, None, None) == 1
    d.ns = 64  # 64 * 128 * 128 cells > the fixed grid capacity
    assert L.ffa_sc_step_static(ctypes.byref(d), ctypes.byref(b.soa()), b.n, 0, 1, s, None, None) == 4
    d.ns = 16
    d.hockney = 1
    assert L.ffa_sc_step_static(ctypes.byref(d), ctypes.byref(b.soa()), b.n, 0, 1, s, None, None) == 4
