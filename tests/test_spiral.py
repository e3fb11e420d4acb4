"""Spiral RF gaps (FFAG_EField_spiral, src/FFAG_Field.py:379-550; the field
lookup interpolate_spiral_emap_unique_gap_kernel, src/FFAG_MathTools.py:
1042-1114: the first gap whose window holds the particle, bilinear in
(r, phi) with linear extrapolation outside the r axis, E = V0 / gap_width *
(Er, Ez/z * z, Ephi) * sin(RF phase + rf_shift)).  The golden vectors come
from the reference's own code (tests/golden/make_golden.py --spiral): its
field lookup on 4000 scattered points (both gaps, their overlap, misses, r
beyond the map), Boris and RK4 single steps and loops through the gaps.

CPU: the oracle reproduces the lookup and the single steps bit for bit and
the loops to the ulp level; the host class reads the reference's files.
GPU: the product's pushers against the same vectors (1e-14 per step, 1e-12
over the loops, flags exact)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.fixtures import load_golden_spiral


@pytest.fixture(scope="module")
def sgold():
    return load_golden_spiral()


@pytest.fixture(scope="module")
def setup(sgold):
    gp = sgold.gp()
    return O.Setup(gp.Bmap, gp.Emap, gp)


def test_host_class_reads_the_reference_files(sgold):
    em = sgold.emap()
    cfg = json.loads(bytes(sgold["spiral_json"]).decode())
    assert em.GapType == "spiral" and em.Er_map.shape == (cfg["r_axis"][2], cfg["nphi"])
    assert np.allclose(np.rad2deg(em.gap_azimuths), cfg["gap_azimuth_deg"], rtol=0, atol=1e-13)
    assert em.acc_Etot_uniform == 1.0 / cfg["gap_width"]
    assert em.dr == em.r_axis[1] - em.r_axis[0] and em.nphi == len(em.phi_axis)
    # the gap-crossing tables interpolate linearly, as np.interp does
    mid = 0.5 * (em.Ek_gap[3] + em.Ek_gap[4])
    assert em.r_gap_interp(mid) == pytest.approx(0.5 * (em.r_gap[3] + em.r_gap[4]), rel=1e-15)
    assert np.all(np.diff(em.Ek_gap) > 0)


def test_oracle_lookup_bit_exact(sgold, setup):
    p = sgold["lookup_in"]
    er, ez, ef, hit = O.spiral_lookup(setup, sgold["lookup_v0"][0] / sgold.emap().gap_width, p[:, 0], p[:, 1],
                                      p[:, 2])
    assert np.array_equal(hit, sgold["lookup_hit"])
    assert np.array_equal(np.stack([er, ez, ef], 1), sgold["lookup_out"])


def test_fixture_exercises_both_gaps_misses_and_extrapolation(sgold):
    hit, p = sgold["lookup_hit"], sgold["lookup_in"]
    em = sgold.emap()
    assert (hit == -1).sum() > 100 and (hit == 0).sum() > 100 and (hit == 1).sum() > 100
    outside = (p[:, 0] < em.map_rmin) | (p[:, 0] > em.map_rmax)
    assert ((hit >= 0) & outside).sum() > 10
    # points inside gap 1's window that gap 0's window also holds go to gap 0
    sh = lambda d: d + 2 * np.pi * np.round((0.5 * (em.map_phimin + em.map_phimax) - d) / (2 * np.pi))
    l0, l1 = sh(p[:, 1] - em.gap_azimuths[0]), sh(p[:, 1] - em.gap_azimuths[1])
    both = (l0 >= em.map_phimin) & (l0 <= em.map_phimax) & (l1 >= em.map_phimin) & (l1 <= em.map_phimax)
    assert both.sum() > 20 and np.all(hit[both] == 0)


def test_oracle_boris_and_rk4_steps_bit_exact(sgold, setup):
    t0, dt = sgold["boris1_t"]
    m = sgold["boris1_in"].copy()
    O.boris_step(setup, m, t0, dt)
    assert np.array_equal(m, sgold["boris1_out"])
    m = sgold["rk41_in"].copy()
    O.rk4_step(setup, m, t0, dt)
    assert np.array_equal(m, sgold["rk41_out"])


@pytest.mark.parametrize("name,solver", [("borisloop", "Boris"), ("rk4loop", "RK4")])
def test_oracle_loops(sgold, setup, name, solver):
    from tests.test_oracle_golden import _check_matrix
    ts, dt, n = sgold[name + "_t"]
    m = sgold[name + "_in"].copy()
    O.track(setup, solver, m, ts, dt, int(n))
    _check_matrix(m, sgold[name + "_out"], 1e-13)


def test_spiral_gap_changes_the_step(sgold):
    """With the RF off the oracle misses the reference's step by far more
    than rounding: the single-step particles sit in the gaps' fields."""
    gp = sgold.gp()
    gp.Emap.EnableFlag = False
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    t0, dt = sgold["boris1_t"]
    m = sgold["boris1_in"].copy()
    O.boris_step(S, m, t0, dt)
    ref = sgold["boris1_out"]
    alive = ref[:, 8] == 1
    assert np.max(np.abs(m[alive, 1] - ref[alive, 1]) / np.abs(ref[alive, 1]).max()) > 1e-6


def test_injection_rf_phase_uses_the_gap_crossing(sgold):
    from pyffa_b200.main_track import calc_injection_rf_phase
    em = sgold.emap()
    Ek, T0 = 300.0, 2.0e-7
    got = calc_injection_rf_phase(em, 0.1, -5e-9, T0, Ek, gap_idx=1)
    phi_gap = em.phi_gap_interp_unwrapped(Ek) + (em.gap_azimuths[1] - em.gap_azimuths[0])
    want = em.acc_phi0 - em.harmonic * (phi_gap - 0.1) - em.harmonic * 2 * np.pi * 5e-9 / T0
    assert got == pytest.approx(want, rel=1e-15)


@pytest.mark.gpu
def test_gpu_pushers_match_reference_with_spiral_gaps(sgold):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    from tests.test_gpu_push import _assert_close
    gp = sgold.gp()
    t0, dt = sgold["boris1_t"]
    m = sgold["boris1_in"].copy()
    FFAG_RungeKutta().Boris_solve(t0, m, dt, GlobalParameters=gp)
    _assert_close(m, sgold["boris1_out"], 1e-14)
    m = sgold["rk41_in"].copy()
    dr, *_ = FFAG_RungeKutta().rk4_step_malloc(None, t0, m, dt, gp)
    _assert_close(m + dr, sgold["rk41_out"], 1e-14)
    for name, solver in (("borisloop", "Boris"), ("rk4loop", "RK4")):
        ts, dt_, n = sgold[name + "_t"]
        b = FFAG_Bunch(sgold[name + "_in"], BunchType=solver)
        lp = {"stop_condition": {"max_stepsN": int(n), "max_turn": 1e9, "max_time": 1e9}, "time_step": dt_,
              "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
        rk = FFAG_RungeKutta(verbose=False)
        getattr(rk, "rk4_solve_dt_bunch3_withSC_boris" if solver == "Boris" else "rk4_solve_dt_bunch3_withSC")(
            None, ts, b, gp, lp)
        _assert_close(b.LocalBunch, sgold[name + "_out"], 1e-12)


@pytest.mark.gpu
def test_gpu_fp32c_and_fp32_through_spiral_gaps(sgold):
    """The float32-field pushers with the spiral gap (the gap itself is
    evaluated in float64 in both): one step against the oracle, within the
    float32 field's error bounds of the FP32C and FP32 single-step tests."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from pyffa_b200.track import FFAG_RungeKutta
    gp = sgold.gp()
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    t0, dt = sgold["boris1_t"]
    ref = sgold["boris1_in"].copy()
    O.boris_step(S, ref, t0, dt)
    for prec, tol in (("fp32c", 1e-9), ("fp32", 1e-5)):
        m = sgold["boris1_in"].copy()
        FFAG_RungeKutta(precision=prec).Boris_solve(t0, m, dt, GlobalParameters=gp)
        assert np.array_equal(m[:, 7:9], ref[:, 7:9])
        alive = ref[:, 8] == 1
        for c in (0, 4):
            assert np.max(np.abs(m[alive, c] - ref[alive, c]) / np.abs(ref[alive, c])) < tol, (prec, c)
        for c in (1, 3):
            assert np.max(np.abs(m[alive, c] - ref[alive, c])) < tol * np.abs(ref[alive, c]).max() * 1e3, (prec, c)
