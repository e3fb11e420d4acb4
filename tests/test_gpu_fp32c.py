"""The FP32C Boris pusher (float32 field exponentials and map lookup,
float64 push) against the float64 one; the RK4 pusher with the same field
against float64 RK4.

Both push the same seeded 6D Gaussian bunch through the full 1301 x 6000 map
(z-Taylor order 2) for 1000 turns at 2880 steps per turn (at 720 steps/turn
the 2.8-degree D magnet is sampled so coarsely that the motion is weakly
chaotic and a single-ulp difference grows without bound, which would
measure the lattice, not the arithmetic).

The runs are compared where the particles cross one azimuth in the last turn
(azimuth-crossing records, state interpolated to the exact azimuth), so that
a tiny difference of the azimuthal speed does not show up as a radius
difference on the scalloped orbit.  Errors: radius |dr|/r, arrival time
|dt|/t (the azimuth error per unit azimuth), momentum |dp|/p, the rms
emittances; z, vr and vz relative to their amplitude.

The scale they are held to is the float64 pusher's own response to a
float32-sized change of the input: the same bunch with every initial radius
multiplied by 1 + 2^-24.  The large-amplitude particles of the bunch (up to
4 cm vertically) have amplitude-dependent tunes, so any change of that size
dephases them; with the RF on, the reference's gap model (a particle is
kicked with the full gap field iff its step lands inside the gap rectangle)
turns a sub-micron change of the arrival position into a whole step more or
less of kick.  Bars: every error within 4 times that response, and without
RF the arrival time, momentum and emittances within 1e-6, 1e-6 and 1 %.
"""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SPT = 2880
TURNS = 1000
KEYS = ("r", "t", "p", "vr_amp", "z_amp", "vz_amp", "emit_x", "emit_z")


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


def _track(gp, v, dt, nsteps, precision, target=None):
    """Tracks a Boris v-format bunch; with `target` (rad) a crossing dump
    over the last 0.85 turn records where each particle passes it."""
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.dump import Dumps, PositionDumpBunch
    from pyffa_b200.track import FFAG_RungeKutta
    b = FFAG_Bunch(v, BunchType="Boris")
    dumps = Dumps()
    d = None
    if target is not None:
        d = PositionDumpBunch(np.rad2deg(target), (nsteps - 0.9 * SPT) * dt, (nsteps - 0.05 * SPT) * dt,
                              save_folder=os.path.join(tempfile.mkdtemp(), "x"))
        dumps.add_dump(d)
    lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": dumps}
    FFAG_RungeKutta(precision=precision, verbose=False).rk4_solve_dt_bunch3_withSC_boris(None, 0.0, b, gp, lp)
    return b.LocalBunch, d


def at_azimuth(d, n, dt):
    """Per particle (NaN where it did not cross): r, vr, z, vz interpolated
    to the target azimuth, the post-step speed and the crossing time."""
    from pyffa_b200 import diagnostics
    rec = d.crossing_records
    idx = rec[:, 1].astype(np.int64)
    assert np.unique(idx).size == idx.size, "one crossing per particle in the window"
    return diagnostics.at_azimuth(rec, n, dt)


def azimuth_errors(s64, s32):
    """Errors of s32 against s64 (rows of at_azimuth)."""
    from pyffa_b200 import diagnostics
    return diagnostics.azimuth_errors(s64, s32)


def _bunch(seed, n=2048):
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    p = synthetic.centred_bunch(n, seed=seed)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 9] = 0.4
    target = (np.mean(v[:, 4]) + np.pi) % (2 * np.pi)   # half a turn from the bunch
    return v, target


def _compare(rf_on):
    from pyffa_b200 import synthetic
    gp = _lattice(rf_on)
    v, target = _bunch(13)
    dt = synthetic.design_dt(300.0, SPT)
    v32 = v.copy()
    v32[:, 0] = v32[:, 0] * (1 + 2.0 ** -24)
    s = {}
    ends = {}
    for name, prec, vin in (("fp64", "fp64", v), ("fp32c", "fp32c", v), ("fp64_r32", "fp64", v32)):
        a, d = _track(gp, vin, dt, TURNS * SPT, prec, target)
        ends[name] = a
        s[name] = at_azimuth(d, v.shape[0], dt)
    return azimuth_errors(s["fp64"], s["fp32c"]), azimuth_errors(s["fp64"], s["fp64_r32"]), ends


def test_fp32c_matches_fp64_after_1000_turns_rf_off():
    e, scale, ends = _compare(False)
    print("\nRF off, fp32c vs fp64 at the azimuth after 1000 turns:", e)
    print("RF off, fp64 response to r * (1 + 2^-24):", scale)
    assert np.array_equal(ends["fp64"][:, 7:9], ends["fp32c"][:, 7:9]) and e["n"] > 1700
    for k in KEYS:
        assert e[k] <= 4 * scale[k], (k, e[k], scale[k])
    assert e["t"] <= 1e-6 and e["p"] <= 1e-6, e
    assert e["emit_x"] <= 0.01 and e["emit_z"] <= 0.01, e


def test_fp32c_with_rf_after_1000_turns():
    e, scale, _ = _compare(True)
    print("\nRF on, fp32c vs fp64 at the azimuth after 1000 turns:", e)
    print("RF on, fp64 response to r * (1 + 2^-24):", scale)
    assert e["n"] > 1700
    for k in KEYS:
        assert e[k] <= 4 * scale[k], (k, e[k], scale[k])


def test_fp32c_single_turn_close_to_fp64():
    """One turn at the benchmark's 720 steps/turn: radius, azimuth and speed
    within 4 times the float64 response to r * (1 + 2^-24) and within 1e-7."""
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    gp = _lattice(True)
    p = synthetic.centred_bunch(4096, seed=17)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v32 = v.copy()
    v32[:, 0] = v32[:, 0] * (1 + 2.0 ** -24)
    dt = synthetic.design_dt(300.0, 720)
    a64, _ = _track(gp, v, dt, 720, "fp64")
    a32, _ = _track(gp, v, dt, 720, "fp32c")
    ar, _ = _track(gp, v32, dt, 720, "fp64")
    assert np.array_equal(a64[:, 7:9], a32[:, 7:9])
    al = a64[:, 8] == 1
    speed = lambda a: np.sqrt(a[:, 1] ** 2 + a[:, 3] ** 2 + (a[:, 0] * a[:, 5]) ** 2)
    for name, f in (("r", lambda a: a[al, 0]), ("fi", lambda a: a[al, 4]), ("v", lambda a: speed(a[al]))):
        err = np.max(np.abs(f(a32) - f(a64)) / np.abs(f(a64)))
        scale = np.max(np.abs(f(ar) - f(a64)) / np.abs(f(a64)))
        print(f"\none turn, {name}: fp32c {err:.3g}, fp64 response to r * (1 + 2^-24) {scale:.3g}")
        assert err <= 1e-7 and err <= max(4 * scale, 1e-12), (name, err, scale)


def test_fp32c_rk4_single_turn_close_to_fp64():
    """The RK4 pusher with the FP32C field (float32 flutter exponentials and
    map lookup; equations of motion and RK4 stages in float64), one turn at
    720 steps per turn with the RF on, against the float64 RK4 pusher:
    flags exact; radius, azimuth and total energy within 1e-7 and within 4
    times the float64 RK4 response to r * (1 + 2^-24); and not bit-equal to
    float64 (the float32 field is the one in use)."""
    from pyffa_b200 import synthetic
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.constants import FFAG_ConversionTools
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    gp = _lattice(True)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek(synthetic.centred_bunch(4096, seed=19))
    dt = synthetic.design_dt(300.0, 720)

    def run(m, precision):
        b = FFAG_Bunch(m.copy(), BunchType="RK4")
        lp = {"stop_condition": {"max_stepsN": 720, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
              "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
        FFAG_RungeKutta(precision=precision, verbose=False).rk4_solve_dt_bunch3_withSC(None, 0.0, b, gp, lp)
        return b.LocalBunch

    v32 = v.copy()
    v32[:, 0] = v32[:, 0] * (1 + 2.0 ** -24)
    a64, a32, ar = run(v, "fp64"), run(v, "fp32c"), run(v32, "fp64")
    assert np.array_equal(a64[:, 7:9], a32[:, 7:9])
    al = a64[:, 8] == 1
    assert al.sum() > 4000
    differs = False
    for name, c in (("r", 0), ("fi", 4), ("E", 5)):
        err = np.max(np.abs(a32[al, c] - a64[al, c]) / np.abs(a64[al, c]))
        scale = np.max(np.abs(ar[al, c] - a64[al, c]) / np.abs(a64[al, c]))
        print(f"\none RK4 turn, {name}: fp32c {err:.3g}, fp64 response to r * (1 + 2^-24) {scale:.3g}")
        assert err <= 1e-7 and err <= max(4 * scale, 1e-12), (name, err, scale)
        differs |= err > 0
    assert differs


def test_fp32_push_single_turn():
    """The float32 pusher (float32 field and push, r, fi, z and the RF phase
    accumulated in float64), one turn at 720 steps/turn against float64:
    flags exact, radius, azimuth and speed within 1e-5 (its float32
    velocities round at ~6e-8 per step), and visibly not float64."""
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    from pyffa_b200.track import Pusher
    from pyffa_b200.bunch import FFAG_Bunch
    gp = _lattice(True)
    p = synthetic.centred_bunch(4096, seed=17)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    dt = synthetic.design_dt(300.0, 720)
    a64, _ = _track(gp, v, dt, 720, "fp64")
    a32, _ = _track(gp, v, dt, 720, "fp32")
    assert np.array_equal(a64[:, 7:9], a32[:, 7:9])
    al = a64[:, 8] == 1
    speed = lambda a: np.sqrt(a[:, 1] ** 2 + a[:, 3] ** 2 + (a[:, 0] * a[:, 5]) ** 2)
    errs = {}
    for name, f in (("r", lambda a: a[al, 0]), ("fi", lambda a: a[al, 4]), ("v", lambda a: speed(a[al]))):
        errs[name] = float(np.max(np.abs(f(a32) - f(a64)) / np.abs(f(a64))))
    print("\none turn, fp32 push vs fp64:", errs)
    assert all(np.isfinite(a32[al, c]).all() for c in range(6))
    assert max(errs.values()) <= 1e-5 and max(errs.values()) > 1e-12, errs
    with pytest.raises(NotImplementedError):
        Pusher(FFAG_Bunch(v.copy(), BunchType="RK4"), gp, "RK4", "fp32")
