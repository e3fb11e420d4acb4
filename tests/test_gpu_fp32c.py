"""The compensated float32 Boris pusher against the float64 one.

Both push the same seeded 6D Gaussian bunch through the full 1301 x 6000 map
(z-Taylor order 2) with the RF gaps on, for 1000 turns at 2880 steps per
turn (at 720 steps/turn the 2.8-degree D magnet is sampled so coarsely that
the motion is weakly chaotic and a single-ulp difference grows without bound,
which would measure the lattice, not the arithmetic).

Stated errors after 1000 turns, relative to each coordinate's own scale:
radius |dr|/r, azimuth |dfi|/fi, momentum |dp|/p and the rms emittances;
the betatron coordinates z, vr, vz are reported relative to their amplitude.
Bars: 1e-6 for r, fi and p; 1 % for the emittances (RF off).  With the RF
on the motion itself amplifies rounding differences; the bar there is the
float64 pusher's own sensitivity to a one-ulp change of its input.
"""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _lattice(rf_on):
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    cfg = synthetic.lattice_bmap()
    bm = FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2))
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=rf_on)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    gp.AddAperture(7.5, 9.5, -0.1, 0.1)
    return gp


@pytest.fixture(scope="module")
def lattice():
    return _lattice(True)


@pytest.fixture(scope="module")
def lattice_no_rf():
    return _lattice(False)


def _track(gp, v, dt, nsteps, precision):
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    b = FFAG_Bunch(v, BunchType="Boris")
    lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
    FFAG_RungeKutta(precision=precision, verbose=False).rk4_solve_dt_bunch3_withSC_boris(None, 0.0, b, gp, lp)
    return b.LocalBunch


def _emittance(x, xp):
    x = x - x.mean()
    xp = xp - xp.mean()
    return np.sqrt(np.mean(x * x) * np.mean(xp * xp) - np.mean(x * xp) ** 2)


def fp32c_errors(a64, a32):
    from pyffa_b200.constants import FFAG_ConversionTools
    c = FFAG_ConversionTools()
    p64, p32 = c.ConvertVrzek2Przek_boris(a64), c.ConvertVrzek2Przek_boris(a32)
    alive = (a64[:, 8] == 1) & (a32[:, 8] == 1)
    mom = lambda a: np.sqrt(a[:, 1] ** 2 + a[:, 3] ** 2 + (a[:, 0] * a[:, 5]) ** 2)
    e = {
        "r": float(np.max(np.abs(a32[alive, 0] - a64[alive, 0]) / a64[alive, 0])),
        "fi": float(np.max(np.abs(a32[alive, 4] - a64[alive, 4]) / np.abs(a64[alive, 4]))),
        "p": float(np.max(np.abs(mom(a32[alive]) - mom(a64[alive])) / mom(a64[alive]))),
    }
    for name, col in (("vr", 1), ("z", 2), ("vz", 3)):
        e[name + "_amp"] = float(np.abs(a32[alive, col] - a64[alive, col]).max() / np.abs(a64[alive, col]).max())
    for name, (cx, cxp) in (("emit_x", (0, 1)), ("emit_z", (2, 3))):
        e64 = _emittance(p64[alive, cx], p64[alive, cxp])
        e32 = _emittance(p32[alive, cx], p32[alive, cxp])
        e[name] = float(abs(e32 - e64) / e64)
    e["alive"] = int(alive.sum())
    e["flags_equal"] = bool(np.array_equal(a64[:, 7:9], a32[:, 7:9]))
    return e


def _bunch(seed):
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    p = synthetic.centred_bunch(2048, seed=seed)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 9] = 0.4
    return v


def test_fp32c_matches_fp64_after_1000_turns(lattice_no_rf):
    """Betatron motion without RF: the float32 increments stay within the bars."""
    from pyffa_b200 import synthetic
    v = _bunch(13)
    spt = 2880
    dt = synthetic.design_dt(300.0, spt)
    nsteps = 1000 * spt
    a64 = _track(lattice_no_rf, v, dt, nsteps, "fp64")
    a32 = _track(lattice_no_rf, v, dt, nsteps, "fp32c")
    e = fp32c_errors(a64, a32)
    print("fp32c vs fp64 after 1000 turns, RF off:", e)
    assert e["flags_equal"] and e["alive"] > 1900
    assert e["r"] <= 1e-6 and e["fi"] <= 1e-6 and e["p"] <= 1e-6, e
    assert e["emit_x"] <= 0.01 and e["emit_z"] <= 0.01, e


def test_fp32c_with_rf_within_fp64_sensitivity(lattice):
    """With the RF gaps on, a gap-crossing timing difference turns into a
    different energy kick, so the motion amplifies any rounding difference.
    The float64 pusher against itself with r nudged by one ulp gives that
    sensitivity; the float32 pusher must stay within 10 times it."""
    from pyffa_b200 import synthetic
    v = _bunch(13)
    spt = 2880
    dt = synthetic.design_dt(300.0, spt)
    nsteps = 1000 * spt
    a64 = _track(lattice, v, dt, nsteps, "fp64")
    vp = v.copy()
    vp[:, 0] = np.nextafter(vp[:, 0], np.inf)
    a64p = _track(lattice, vp, dt, nsteps, "fp64")
    a32 = _track(lattice, v, dt, nsteps, "fp32c")
    floor = fp32c_errors(a64, a64p)
    e = fp32c_errors(a64, a32)
    print("RF on, fp64 one-ulp sensitivity:", floor)
    print("RF on, fp32c vs fp64:", e)
    for k in ("r", "fi", "p", "emit_x", "emit_z"):
        assert e[k] <= max(1e-6, 10 * floor[k]), (k, e[k], floor[k])


def test_fp32c_single_turn_close_to_fp64(lattice):
    """One turn at the benchmark's 720 steps/turn: float32 increments keep the
    radius and momentum within 1e-8 of the float64 result."""
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    p = synthetic.centred_bunch(4096, seed=17)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    dt = synthetic.design_dt(300.0, 720)
    a64 = _track(lattice, v, dt, 720, "fp64")
    a32 = _track(lattice, v, dt, 720, "fp32c")
    e = fp32c_errors(a64, a32)
    assert e["flags_equal"]
    assert e["r"] <= 1e-8 and e["p"] <= 1e-8 and e["fi"] <= 1e-8, e
