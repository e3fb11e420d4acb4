"""Field-error harmonics (FFAG_BField_Error, src/FFAG_Field.py:947-1042):
Bz += sum_k A_k cos(m_k fi + phase_k) inside each harmonic's radial band,
added after the map by Boris_solve (src/FFAG_track.py:1007) and the RK4 field
function (:1782).  The golden vectors come from the reference's own code with
harmonics enabled (tests/golden/make_golden.py --harmonics).

CPU: the oracle reproduces the reference's single steps bit for bit and its
loops to the ulp level; the host class matches the reference's parameters.
GPU: the product's pushers against the same vectors (1e-14 per step, 1e-12
over the loops, flags exact) and against the oracle without harmonics, which
they must differ from."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from tests.fixtures import load_golden_harmonics


@pytest.fixture(scope="module")
def hgold():
    return load_golden_harmonics()


@pytest.fixture(scope="module")
def setup(hgold):
    gp = hgold.gp()
    return O.Setup(gp.Bmap, gp.Emap, gp)


def test_host_class_matches_reference_parameters(hgold):
    from pyffa_b200.fields import FFAG_BField_Error
    cfg = json.loads(bytes(hgold["harmonics_json"]).decode())
    h = FFAG_BField_Error(cfg, True)
    assert h.active() and h.Nharm == len(cfg)
    assert np.array_equal(h.m_arr, [c["m"] for c in cfg])
    assert np.allclose(h.amp_arr, [c["amp_Gs"] * 1e-4 for c in cfg], rtol=0, atol=0)
    assert np.allclose(h.phase_arr, np.deg2rad([c["phase_deg"] for c in cfg]), rtol=0, atol=0)
    r = np.array([8.05, 8.2, 8.55])
    bz = h.GetBzHarmonics(r, 0.3)
    want = [sum(c["amp_Gs"] * 1e-4 * np.cos(c["m"] * 0.3 + np.deg2rad(c["phase_deg"]))
                for c in cfg if c["rmin"] <= rr <= c["rmax"]) for rr in r]
    assert np.allclose(bz, want, rtol=1e-15, atol=0)
    assert not FFAG_BField_Error(cfg, False).active()


def test_oracle_boris_and_rk4_steps_bit_exact(hgold, setup):
    t0, dt = hgold["boris1_t"]
    m = hgold["boris1_in"].copy()
    O.boris_step(setup, m, t0, dt)
    assert np.array_equal(m, hgold["boris1_out"])
    m = hgold["rk41_in"].copy()
    O.rk4_step(setup, m, t0, dt)
    assert np.array_equal(m, hgold["rk41_out"])


@pytest.mark.parametrize("name,solver", [("borisloop", "Boris"), ("rk4loop", "RK4")])
def test_oracle_loops(hgold, setup, name, solver):
    from tests.test_oracle_golden import _check_matrix
    ts, dt, n = hgold[name + "_t"]
    m = hgold[name + "_in"].copy()
    O.track(setup, solver, m, ts, dt, int(n))
    _check_matrix(m, hgold[name + "_out"], 1e-13)


def test_harmonics_change_the_step(hgold):
    """Without the harmonics the oracle misses the reference's step by far
    more than rounding: the fixture exercises them."""
    gp = hgold.gp()
    gp.BHarmonics = None
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    t0, dt = hgold["boris1_t"]
    m = hgold["boris1_in"].copy()
    O.boris_step(S, m, t0, dt)
    ref = hgold["boris1_out"]
    alive = ref[:, 8] == 1
    assert np.max(np.abs(m[alive, 1] - ref[alive, 1]) / np.abs(ref[alive, 1]).max()) > 1e-6


@pytest.mark.gpu
def test_gpu_pushers_match_reference_with_harmonics(hgold):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    from tests.test_gpu_push import _assert_close
    gp = hgold.gp()
    t0, dt = hgold["boris1_t"]
    m = hgold["boris1_in"].copy()
    FFAG_RungeKutta().Boris_solve(t0, m, dt, GlobalParameters=gp)
    _assert_close(m, hgold["boris1_out"], 1e-14)
    m = hgold["rk41_in"].copy()
    dr, *_ = FFAG_RungeKutta().rk4_step_malloc(None, t0, m, dt, gp)
    _assert_close(m + dr, hgold["rk41_out"], 1e-14)
    for name, solver in (("borisloop", "Boris"), ("rk4loop", "RK4")):
        ts, dt_, n = hgold[name + "_t"]
        b = FFAG_Bunch(hgold[name + "_in"], BunchType=solver)
        lp = {"stop_condition": {"max_stepsN": int(n), "max_turn": 1e9, "max_time": 1e9}, "time_step": dt_,
              "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
        rk = FFAG_RungeKutta(verbose=False)
        getattr(rk, "rk4_solve_dt_bunch3_withSC_boris" if solver == "Boris" else "rk4_solve_dt_bunch3_withSC")(
            None, ts, b, gp, lp)
        _assert_close(b.LocalBunch, hgold[name + "_out"], 1e-12)
