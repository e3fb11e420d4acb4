"""Pins the CPU oracle to the reference: golden vectors produced by running
PyFFA's own Numba kernels (tests/golden/make_golden.py) must be reproduced.

The Boris and RK4 single steps are bit-exact; loops of a few hundred steps
agree to a few ulp (the reference's high-order map sum is compiled with
fastmath, which lets LLVM fuse multiply-adds).  The space-charge cube and slice
indices are bit-exact; potentials and fields differ only by the transforms'
precision (reference: complex64 FFT; oracle: float64).  The fields are
central differences of a float32 potential, so their error is bounded by a
few float32 ulp of max|phi| over the cell size (field_tol below).
"""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def setup(golden):
    gp = golden.gp()
    return O.Setup(gp.Bmap, gp.Emap, gp)


def _check_matrix(m, ref, rtol):
    # flags and identifiers exactly, coordinates to rtol
    assert np.array_equal(m[:, 7:9], ref[:, 7:9])
    assert np.array_equal(m[:, 6], ref[:, 6]) and np.array_equal(m[:, 13:], ref[:, 13:])
    for c in (0, 1, 2, 3, 4, 5, 9, 10, 11, 12):
        scale = np.maximum(np.abs(ref[:, c]), np.abs(ref[:, c]).max() * 1e-6 + 1e-300)
        err = np.max(np.abs(m[:, c] - ref[:, c]) / scale)
        assert err <= rtol, f"column {c}: relative error {err:.3g} > {rtol}"


def test_boris_single_step_bit_exact(golden, setup):
    t0, dt = golden["boris1_t"]
    m = golden["boris1_in"].copy()
    O.boris_step(setup, m, t0, dt)
    assert np.array_equal(m, golden["boris1_out"])


def test_golden_exercises_loss_rf_and_skipped(golden):
    a, b = golden["boris1_in"], golden["boris1_out"]
    assert ((a[:, 8] == 1) & (b[:, 8] == 0)).sum() >= 3          # aperture losses
    assert (a[:, 7] == 0).sum() >= 4                              # not-injected particles
    bl = golden["borisloop_out"]
    assert (bl[:, 7] == 1).all() and (bl[:, 8] == 0).any() and (bl[:, 8] == 1).any()


def test_rk4_single_step_bit_exact(golden, setup):
    t0, dt = golden["boris1_t"]
    m = golden["rk41_in"].copy()
    O.rk4_step(setup, m, t0, dt)
    assert np.array_equal(m, golden["rk41_out"])


@pytest.mark.parametrize("name,solver", [("borisloop", "Boris"), ("rk4loop", "RK4")])
def test_tracking_loop_with_injection(golden, setup, name, solver):
    ts, dt, n = golden[name + "_t"]
    m = golden[name + "_in"].copy()
    O.track(setup, solver, m, ts, dt, int(n))
    _check_matrix(m, golden[name + "_out"], 1e-13)


def test_space_charge_update(golden):
    ns, nx, nz, sr, qm = golden["sc_params"]
    seo = dict(golden.seo)
    seo["pr"] = seo["pr"] + golden["seo_pr_offset"][0]
    m = golden["sc_in"].copy()
    alive = m[:, 8] != 0
    res = O.sc_step(m, alive, seo, int(ns), int(nx), int(nz), sr, qm)
    d = res["diag"]
    box = golden["sc_box"]
    got = [d["xmin"], d["xmax"], d["zmin"], d["zmax"], d["bunch_length"], d["fi_s"], d["fi_e"]]
    np.testing.assert_allclose(got, box, rtol=1e-13, atol=1e-15)
    assert np.array_equal(res["rho"], golden["sc_rho"])
    assert np.array_equal(res["slice_idx"][alive], golden["sc_slice_indices"])
    ref_phi = golden["sc_phi"]
    assert np.abs(res["phi"] - ref_phi).max() <= 2e-6 * np.abs(ref_phi).max()
    tol = field_tol(ref_phi, golden["sc_ex"], golden["sc_ez"], d["dx"], d["dz"])
    for k in ("ex", "ez"):
        assert np.abs(res[k] - golden["sc_" + k]).max() <= tol, k
    ref = golden["sc_out"]
    for c in (10, 11, 12):
        assert np.abs(m[:, c] - ref[:, c]).max() <= tol, c
    assert np.array_equal(m[~alive], golden["sc_in"][~alive])


def field_tol(phi, ex, ez, dx, dz):
    """Field error bound: 8 float32 ulp of max|phi| per cell, plus 2e-6 of max|E|."""
    eps32 = float(np.finfo(np.float32).eps)
    emax = max(np.abs(ex).max(), np.abs(ez).max())
    return 8 * eps32 * float(np.abs(phi).max()) / min(dx, dz) + 2e-6 * emax


def sc_loop(setup, mat, t_start, dt, nsteps, sc_step, seo, grid, q_macro, solver="Boris"):
    """The reference step loop with space charge (src/FFAG_track.py:297-579),
    restated on the oracle's primitives."""
    N = mat.shape[0]
    pre = np.zeros(N, bool)
    pp = np.zeros(N, bool)
    e_pre = np.zeros((N, 3))
    e_pp = np.zeros((N, 3))
    head = np.zeros(1, np.int64)
    t = t_start
    import ctypes
    h = ctypes.c_int64(0)
    for s in range(nsteps):
        O.lib().orc_inject(mat.ctypes.data, N, t, dt, ctypes.byref(h))
        if s % sc_step == 0:
            alive = mat[:, 8] != 0
            O.sc_step(mat, alive, seo, grid[0], grid[1], grid[2], grid[3], q_macro, boris=(solver == "Boris"))
            if s == 0:
                pre[:] = alive
                pp[:] = False
                e_pre[alive] = mat[alive, 10:13]
                e_pp[:] = e_pre
            else:
                pp[:] = pre
                pre[:] = alive
                e_pp[:] = e_pre
                e_pre[alive] = mat[alive, 10:13]
        k = s % sc_step
        sf = k / sc_step if s >= sc_step else 0.0
        both = pre & pp
        only = pre & ~pp
        ep = np.zeros((N, 3))
        ep[both] = e_pre[both] + sf * (e_pre[both] - e_pp[both])
        ep[only] = e_pre[only]
        mat[pre, 10:13] = ep[pre]
        if solver == "Boris":
            O.boris_step(setup, mat, t, dt)
        else:
            O.rk4_step(setup, mat, t, dt)
        t = t + dt
    return mat


def test_space_charge_loop(golden, setup):
    ts, dt, n, sc_step, marco = golden["scloop_t"]
    m = golden["scloop_in"].copy()
    sc_loop(setup, m, ts, dt, int(n), int(sc_step), golden.seo, (8, 32, 32, 6.0), marco * 1.60217662e-19)
    ref = golden["scloop_out"]
    assert np.array_equal(m[:, 7:9], ref[:, 7:9])
    # The reference's float32 field noise (see field_tol) reaches the
    # coordinates through the kicks, and a particle whose azimuth sits on a
    # slice boundary can land in the neighbouring slice.  So: 99 % of the
    # particles within a tight bound per column, every particle within a loose
    # one (a plumbing error in the masks or the extrapolation is O(1)).
    for c, tol in ((0, 1e-7), (4, 1e-7), (1, 1e-5), (5, 1e-6), (2, 1e-4), (3, 1e-4)):
        d = np.abs(m[:, c] - ref[:, c]) / np.abs(ref[:, c]).max()
        assert np.quantile(d, 0.99) <= tol and d.max() <= 1e-2, c
    for c in (10, 11, 12):
        d = np.abs(m[:, c] - ref[:, c]) / np.abs(ref[:, c]).max()
        assert np.quantile(d, 0.99) <= 5e-3 and d.max() <= 0.2, c


def test_rounding_noise_run(golden, setup):
    """orc_track_noisy (the rounding-sensitivity measure of the long GPU
    parity tests): one step is the plain step with each of r, vr, z, vz, fi
    and f5 at most one ulp away, flags and the other columns untouched; the
    same seed and first step repeat exactly, another seed differs."""
    ts, dt, _ = golden["borisloop_t"]
    m0 = golden["borisloop_in"].copy()
    plain, a, b, c = m0.copy(), m0.copy(), m0.copy(), m0.copy()
    O.track(setup, "Boris", plain, ts, dt, 1)
    O.track(setup, "Boris", a, ts, dt, 1, noise=(7, 0))
    O.track(setup, "Boris", b, ts, dt, 1, noise=(7, 0))
    O.track(setup, "Boris", c, ts, dt, 1, noise=(8, 0))
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.array_equal(a[:, 6:], plain[:, 6:])
    d = a[:, :6] != plain[:, :6]
    assert 0.3 < d.mean() < 0.7
    assert np.array_equal(np.nextafter(plain[:, :6], a[:, :6])[d], a[:, :6][d])
