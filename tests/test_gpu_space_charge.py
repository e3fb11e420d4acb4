"""Parity of the CUDA 2.5D space-charge update with the reference and the oracle.

What is exact and what is a tolerance:
- slice indices and deposit cell indices: exact (integer work);
- the bunch box, arc and bunch length: float64 reductions in a different
  order than the reference's serial loop, 1e-12 relative;
- the charge cube: the device sums fixed-point weights exactly while the
  reference accumulates float32 in particle order, so the cube agrees to the
  reference's float32 accumulation error (1e-6 of the maximum);
- potential and fields: float32 FFTs on both sides (FFTW complex64 in the
  reference); fields within a few float32 ulp of max|phi| per cell
  (field_tol in test_oracle_golden).
"""
import numpy as np
import pytest

from tests.test_oracle_golden import field_tol

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _bunch(mat, grid, marco, seo, bunch_type="Boris"):
    from pyffa_b200.bunch import FFAG_Bunch
    b = FFAG_Bunch(mat, marcosize=marco, sc_grid_size=grid, BunchType=bunch_type)
    b.SEO_fi_axis, b.SEO_Ek_axis = seo["fi_axis"], seo["Ek_axis"]
    b.SEO_r_matrix, b.SEO_pr_matrix, b.SEO_perimeter = seo["r"], seo["pr"], seo["perimeter"]
    return b


def test_update_matches_reference_golden(golden):
    from pyffa_b200.space_charge import SpaceCharge
    ns, nx, nz, sr, qm = golden["sc_params"]
    seo = dict(golden.seo)
    seo["pr"] = seo["pr"] + golden["seo_pr_offset"][0]
    m_in = golden["sc_in"]
    b = _bunch(m_in, (int(ns), int(nx), int(nz), sr), qm / 1.60217662e-19, seo)
    sc = SpaceCharge(b)
    sc.update(first=True, roll=False)
    d = sc.diag()
    got = [d["xmin"], d["xmax"], d["zmin"], d["zmax"], d["bunch_length"], d["fi_s"], d["fi_e"]]
    np.testing.assert_allclose(got, golden["sc_box"], rtol=1e-12, atol=1e-15)
    buf = sc.buffers()
    alive = m_in[:, 8] != 0
    assert np.array_equal(buf["slice_idx"][alive], golden["sc_slice_indices"])
    assert (buf["slice_idx"][~alive] == -1).all()
    rho_ref = golden["sc_rho"]
    assert np.abs(buf["rho"] - rho_ref).max() <= 1e-6 * np.abs(rho_ref).max()
    tol = field_tol(golden["sc_phi"], golden["sc_ex"], golden["sc_ez"], d["dx"], d["dz"])
    for k in ("ex", "ez"):
        assert np.abs(buf[k] - golden["sc_" + k]).max() <= tol, k
    out = b.LocalBunch
    ref = golden["sc_out"]
    for c in (10, 11, 12):
        assert np.abs(out[:, c] - ref[:, c]).max() <= tol, c
    assert np.array_equal(out[~alive, 10:13], m_in[~alive, 10:13])


@pytest.fixture(scope="module")
def kv_bunch_1e5():
    from pyffa_b200 import orbit, synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    seo = orbit.seo_tables(synthetic.lattice_bmap(), np.linspace(290.0, 310.0, 9), nfi=361)
    seo = {k: seo[k] for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}
    p = synthetic.centred_bunch(100_000, seed=21, kind="kv", a_x=4e-3, a_z=4e-3, sig_t=20e-9, fi0=np.pi)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    v[:1000, 8] = 0.0
    return v, seo


@pytest.mark.parametrize("hockney", [False, True])
def test_update_vs_oracle_at_size(kv_bunch_1e5, hockney):
    """1e5 KV particles, 64 slices, 128 x 128 grid (256 x 256 doubled when
    open-boundary): per-particle indices exact, cubes and fields to float32."""
    from oracle import oracle as O
    from pyffa_b200.space_charge import SpaceCharge
    v, seo = kv_bunch_1e5
    grid = (64, 128, 128, 12.0)
    marco = 1e13 / v.shape[0]
    b = _bunch(v, grid, marco, seo)
    sc = SpaceCharge(b, hockney=hockney)
    sc.update(first=True, roll=False)
    d = sc.diag()
    buf = sc.buffers()
    m = v.copy()
    ref = O.sc_step(m, m[:, 8] != 0, seo, 64, 128, 128, 12.0, marco * 1.60217662e-19, hockney=hockney)
    rd = ref["diag"]
    # sums over 1e5 particles in a different order than the serial loop; the
    # mean gamma - 1 loses a factor gamma / (gamma - 1) to cancellation
    for k in ("xmin", "xmax", "zmin", "zmax", "bunch_length", "fi_s", "fi_e", "mean_gamma_m1"):
        assert abs(d[k] - rd[k]) <= 1e-11 * max(abs(rd[k]), 1e-3), k
    assert d["count"] == rd["count"] == 99_000
    assert np.array_equal(buf["slice_idx"], ref["slice_idx"])
    # cell indices: exact except particles within 1e-9 of a cell edge, where
    # the box's last-bit difference may move them (none expected)
    diff = buf["cell_idx"] != ref["cell_idx"]
    assert diff.sum() <= 2
    rmax = np.abs(ref["rho"]).max()
    assert np.abs(buf["rho"] - ref["rho"]).max() <= 2e-6 * rmax
    tol = field_tol(ref["phi"], ref["ex"], ref["ez"], rd["dx"], rd["dz"])
    assert np.abs(buf["phi"] - ref["phi"]).max() <= 1e-5 * np.abs(ref["phi"]).max()
    for k in ("ex", "ez"):
        assert np.abs(buf[k] - ref[k]).max() <= 4 * tol, k
    out = b.LocalBunch
    for c in (10, 11, 12):
        assert np.abs(out[:, c] - m[:, c]).max() <= 4 * tol, c


def test_update_is_deterministic(kv_bunch_1e5):
    from pyffa_b200.space_charge import SpaceCharge
    v, seo = kv_bunch_1e5
    outs = []
    for _ in range(2):
        b = _bunch(v, (64, 128, 128, 12.0), 1e8, seo)
        sc = SpaceCharge(b)
        sc.update(first=True, roll=False)
        outs.append((sc.buffers()["rho"], b.LocalBunch[:, 10:13]))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_hockney_round_beam_known_answer():
    """Open-boundary solve of a long uniform round beam: inside, the
    transverse field is E = lambda r / (2 pi eps0 a^2) / gamma^2 (the KV
    linear field the reference's tune-shift benchmarks use,
    benchmarks/Benchmark_SC_analitical.py:51-100)."""
    from pyffa_b200 import orbit, synthetic
    from pyffa_b200.constants import FFAG_ConversionTools, Q
    from pyffa_b200.space_charge import SpaceCharge
    seo = orbit.seo_tables(synthetic.lattice_bmap(), np.linspace(290.0, 310.0, 9), nfi=361)
    seo = {k: seo[k] for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}
    n = 400_000
    rng = np.random.Generator(np.random.PCG64(5))
    a = 4e-3
    rad = a * np.sqrt(rng.uniform(0, 1, n))
    th = rng.uniform(0, 2 * np.pi, n)
    d = synthetic.design(300.0)
    p = np.zeros((n, 16))
    fi = np.pi + rng.uniform(-0.05, 0.05, n)
    fm = fi % (2 * np.pi)
    r0 = np.array([np.interp(f, seo["fi_axis"], seo["r"][4]) for f in fm[:1]])[0]
    p[:, 0] = np.interp(fm, seo["fi_axis"], seo["r"][4]) + rad * np.cos(th)
    p[:, 2] = rad * np.sin(th)
    p[:, 4] = fi
    p[:, 5] = 300.0
    p[:, 15] = np.arange(n)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 7] = v[:, 8] = 1.0
    marco = 1e12 / n
    b = _bunch(v, (16, 128, 128, 6.0), marco, seo)
    sc = SpaceCharge(b, hockney=True)
    sc.update(first=True, roll=False)
    dg = sc.diag()
    out = b.LocalBunch
    gamma = dg["mean_gamma_m1"] + 1.0
    # The reference normalises a slice's charge by bunch_length / ns, while the
    # ns slice boundaries split [fi_s, fi_e] into ns - 1 intervals (the last
    # slice only holds particles at fi_e exactly): the deposited line density
    # of a uniform bunch is ns / (ns - 1) times N q / bunch_length.
    ns = 16
    lam = marco * Q * n / dg["bunch_length"] * ns / (ns - 1)
    x = out[:, 0] - np.interp(fm, seo["fi_axis"], seo["r"][4])
    z = out[:, 2]
    rr = np.hypot(x, z)
    inner = rr < 0.7 * a
    e_theory = lam * rr / (2 * np.pi * 8.854187817e-12 * a * a) / gamma ** 2
    pr0 = np.interp(fm, seo["fi_axis"], seo["pr"][4])
    er = out[:, 10] * np.sqrt(1 + pr0 ** 2)   # undo the projection on the orbit direction
    e_mag = np.hypot(er, out[:, 11])
    rel = np.abs(e_mag[inner] - e_theory[inner]) / (lam * a / (2 * np.pi * 8.854187817e-12 * a * a) / gamma ** 2)
    assert np.median(rel) < 0.03, np.median(rel)
    del r0


def test_tracking_loop_with_sc_matches_reference_golden(golden):
    """The product loop with space charge every 5 steps against the
    reference's own loop (golden): injection, updates, endpoint roll and the
    per-step extrapolation."""
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    ts, dt, n, sc_step, marco = golden["scloop_t"]
    b = _bunch(golden["scloop_in"], (8, 32, 32, 6.0), marco, golden.seo)
    lp = {"stop_condition": {"max_stepsN": int(n), "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": True, "SC_type": 1, "SC_step": int(sc_step), "step_dumps": Dumps()}
    FFAG_RungeKutta(verbose=False).rk4_solve_dt_bunch3_withSC_boris(None, ts, b, golden.gp(), lp)
    m = b.LocalBunch
    ref = golden["scloop_out"]
    assert np.array_equal(m[:, 7:9], ref[:, 7:9])
    for c, tol in ((0, 1e-7), (4, 1e-7), (1, 1e-5), (5, 1e-6), (2, 1e-4), (3, 1e-4)):
        dd = np.abs(m[:, c] - ref[:, c]) / np.abs(ref[:, c]).max()
        assert np.quantile(dd, 0.99) <= tol and dd.max() <= 1e-2, c
    for c in (10, 11, 12):
        dd = np.abs(m[:, c] - ref[:, c]) / np.abs(ref[:, c]).max()
        assert np.quantile(dd, 0.99) <= 5e-3 and dd.max() <= 0.2, c
