"""The c2 cycle on the FP32C pusher against the FP64 one.

One turn of the 2.5D space-charge cycle of the c2 workload (a KV bunch with
4 mm radii and sigma_t = 20 ns at 300 MeV, 1e13 protons, 64 slices on a
128 x 128 grid, open-boundary solve, an update every 60 of the 720 steps per
turn, the field extrapolated in between; src/FFAG_track.py:297-579 with
src/FFAG_Bunch.py:1157-1352), run through the product step loop once with
the compensated float32 pusher and once with the float64 one.  The space-
charge step itself is identical in both runs (same kernels); what differs is
the push, and through the positions, the fields of the later updates.

Exact: injection and loss flags.  Stated against float64, with bars: the
radius, azimuth and momentum of the surviving particles after the turn, the
largest error within 4 times the float64 run's own response to a
float32-sized input change (every initial radius times 1 + 2^-24), and the
median error within the absolute bars below.  The largest errors cannot have
an absolute bar: the 2.5D model gives each particle the field of its slice,
and a particle that the rounding moves across a slice boundary sees another
slice's field, so the response itself reaches 2e-4 of r in one turn for the
particles at the boundaries, while the median stays at the float32 field's
level.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = 20_000


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _setup():
    import os
    import tempfile
    from pyffa_b200 import orbit, synthetic
    from pyffa_b200.constants import FFAG_ConversionTools, FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    cfg = synthetic.lattice_bmap()
    bm = FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2))
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=True)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    gp.AddAperture(7.5, 9.5, -0.1, 0.1)
    t = orbit.seo_tables(cfg, np.linspace(280.0, 320.0, 9), nfi=721)
    seo = {k: t[k] for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}
    p = synthetic.centred_bunch(N, seed=11, kind="kv", a_x=4e-3, a_z=4e-3, sig_t=20e-9, fi0=np.pi)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    return gp, seo, v, synthetic.design_dt(300.0, 720)


def _turn(gp, seo, v, dt, precision):
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    b = FFAG_Bunch(v.copy(), marcosize=1e13 / N, sc_grid_size=(64, 128, 128, 12.0), BunchType="Boris")
    b.SEO_fi_axis, b.SEO_Ek_axis, b.SEO_r_matrix = seo["fi_axis"], seo["Ek_axis"], seo["r"]
    b.SEO_pr_matrix, b.SEO_perimeter = seo["pr"], seo["perimeter"]
    lp = {"stop_condition": {"max_stepsN": 720, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": True, "SC_type": 1, "SC_step": 60, "SC_hockney": True, "step_dumps": Dumps()}
    FFAG_RungeKutta(precision=precision, verbose=False).rk4_solve_dt_bunch3_withSC_boris(None, 0.0, b, gp, lp)
    return b.LocalBunch


def _errors(a, b, alive, c=2.99792458e8, stat=np.max):
    speed = lambda m: np.sqrt(m[:, 1] ** 2 + m[:, 3] ** 2 + (m[:, 0] * m[:, 5]) ** 2)
    mom = lambda m: speed(m) / np.sqrt(1.0 - (speed(m) / c) ** 2)
    return {"r": float(stat(np.abs(b[alive, 0] - a[alive, 0]) / a[alive, 0])),
            "fi": float(stat(np.abs(b[alive, 4] - a[alive, 4]) / np.abs(a[alive, 4]))),
            "p": float(stat(np.abs(mom(b[alive]) - mom(a[alive])) / mom(a[alive])))}


def test_c2_turn_fp32c_vs_fp64():
    gp, seo, v, dt = _setup()
    a64 = _turn(gp, seo, v, dt, "fp64")
    a32 = _turn(gp, seo, v, dt, "fp32c")
    v_r = v.copy()
    v_r[:, 0] *= 1 + 2.0 ** -24
    ar = _turn(gp, seo, v_r, dt, "fp64")
    assert np.array_equal(a64[:, 7], a32[:, 7]), "injection flags"
    assert np.array_equal(a64[:, 8], a32[:, 8]), "loss flags"
    alive = a64[:, 8] == 1
    assert alive.sum() > N // 4
    e = _errors(a64, a32, alive)
    med = _errors(a64, a32, alive, stat=np.median)
    scale = _errors(a64, ar, alive & (ar[:, 8] == 1))
    print("\nc2 turn, fp32c vs fp64: max", e, "median", med, "\nfp64 response to r * (1 + 2^-24):", scale,
          "\nalive fraction:", float(alive.mean()))
    bars = {"r": 1e-6, "fi": 1e-7, "p": 1e-6}
    for k in ("r", "fi", "p"):
        assert e[k] <= max(4 * scale[k], 1e-12), (k, e[k], scale[k])
        assert med[k] <= bars[k], (k, med[k])
