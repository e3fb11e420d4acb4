"""Edge cases of the push and space-charge paths, against the oracle:

- an empty bunch (n = 0, no columns): every call returns without work, a
  space-charge update reports a degenerate grid;
- ragged sizes (1, 31, 33, 4099 particles: partial warps and blocks, the
  Morton order's small-range identity and its permutation);
- every particle lost or not yet injected: the reference still converts
  them to Cartesian and back each step, so they drift by rounding exactly as
  the oracle's;
- a non-finite particle: counted in the NaN status word, its neighbours'
  steps unchanged;
- particles beyond the z-Taylor map's r range: counted as clamped lookups,
  and extrapolated as the reference does;
- a space-charge update whose particles all sit at one point (zero box):
  counted as degenerate, the particles' fields left as they were, no
  fault."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _push(gp, mat, t0, dt, solver="Boris", precision="fp64", steps=1):
    from pyffa_b200.track import Pusher, StepClock, _EphemeralBunch
    dev = torch.device("cuda", 0)
    b = _EphemeralBunch(np.ascontiguousarray(mat), solver, dev)
    clock = StepClock(t0, dt, gp.Emap, solver, dev)
    clock.ensure(steps)
    pu = Pusher(b, gp, solver, precision)
    pu.push(clock, 0, steps, 0)
    torch.cuda.synchronize()
    st = b.status.cpu().numpy()
    return b.matrix(), {"lost": int(st[0]), "nan": int(st[1]), "oob": int(st[2])}


def _close(m, ref, rtol):
    from tests.test_gpu_push import _assert_close
    _assert_close(m, ref, rtol)


def test_empty_bunch(golden):
    from pyffa_b200 import _lib
    from pyffa_b200.track import FFAG_RungeKutta
    gp = golden.gp()
    t0, dt = golden["boris1_t"]
    m = np.zeros((0, 16))
    assert FFAG_RungeKutta().Boris_solve(t0, m, dt, GlobalParameters=gp).shape == (0, 16)
    dr, *_ = FFAG_RungeKutta().rk4_step_malloc(None, t0, m, dt, gp)
    assert dr.shape == (0, 16)
    L = _lib.lib()
    st = _lib.StateSoA()                                          # all columns NULL
    assert L.ffa_aos_to_soa(None, 0, ctypes.byref(st), None) == 0
    assert L.ffa_soa_to_aos(ctypes.byref(st), 0, None, None) == 0


@pytest.mark.parametrize("n", [1, 31, 33, 4099])
def test_ragged_sizes_match_oracle(golden, n):
    gp = golden.gp()
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    t0, dt = golden["boris1_t"]
    base = golden["boris1_in"]
    rng = np.random.default_rng(n)
    m = base[rng.integers(0, base.shape[0], n)].copy()
    m[:, 0] *= 1 + 1e-6 * rng.standard_normal(n)                  # distinct particles
    got, _ = _push(gp, m, t0, dt, steps=1)
    ref = m.copy()
    O.boris_step(S, ref, t0, dt)
    _close(got, ref, 1e-14)


def test_lost_and_uninjected_particles_drift_like_the_oracle(golden):
    gp = golden.gp()
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    t0, dt = golden["boris1_t"]
    m = golden["boris1_in"].copy()
    m[::2, 8] = 0.0           # lost
    m[1::4, 7] = 0.0          # not injected
    got, st = _push(gp, m, t0, dt, steps=1)
    ref = m.copy()
    O.boris_step(S, ref, t0, dt)
    _close(got, ref, 1e-14)
    # the live particles that the oracle loses at the aperture (the fixture
    # puts some outside it) are the ones counted; the others keep their flags
    assert st["lost"] == int(((m[:, 7] == 1) & (m[:, 8] == 1) & (ref[:, 8] == 0)).sum()) > 0
    assert np.array_equal(got[:, 7:9], ref[:, 7:9])


def test_nan_particle_counted_neighbours_unchanged(golden):
    gp = golden.gp()
    t0, dt = golden["boris1_t"]
    m = golden["boris1_in"].copy()
    m[20:24, 7:9] = 1.0
    clean, st0 = _push(gp, m, t0, dt)
    bad = m.copy()
    bad[21, 0] = np.nan
    got, st = _push(gp, bad, t0, dt)
    assert st["nan"] >= 1 and st0["nan"] == 0
    keep = np.arange(m.shape[0]) != 21
    assert np.array_equal(got[keep], clean[keep])


def test_beyond_the_map_counted_and_extrapolated(golden):
    gp = golden.gp(aperture=False)
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    t0, dt = golden["boris1_t"]
    m = golden["boris1_in"].copy()
    m[:, 7:9] = 1.0
    m[:6, 0] = [7.90, 7.95, 7.99, 8.51, 8.55, 8.60]               # the fixture's map covers r 8.0-8.5 m
    got, st = _push(gp, m, t0, dt)
    ref = m.copy()
    O.boris_step(S, ref, t0, dt)
    assert st["oob"] >= 6
    _close(got, ref, 1e-14)


def test_space_charge_on_a_point_bunch_is_degenerate(golden):
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.space_charge import SpaceCharge
    seo = dict(golden.seo)
    m = golden["sc_in"][:64].copy()
    m[:, 7:9] = 1.0
    m[:, 0:6] = m[0, 0:6]                                         # every particle at one point
    b = FFAG_Bunch(m, marcosize=1e9, sc_grid_size=(8, 32, 32, 6.0), BunchType="Boris")
    b.SEO_fi_axis, b.SEO_Ek_axis, b.SEO_r_matrix = seo["fi_axis"], seo["Ek_axis"], seo["r"]
    b.SEO_pr_matrix, b.SEO_perimeter = seo["pr"], seo["perimeter"]
    sc = SpaceCharge(b)
    sc.update(first=True, roll=False)
    torch.cuda.synchronize()
    d = sc.diag()
    assert d["degenerate"] == 1 and d["dx"] == 0.0
    assert b.status_counts()["sc_degenerate"] >= 1
    # no field update for a degenerate grid: the particles keep their fields
    assert np.array_equal(b.LocalBunch[:, 10:13], m[:, 10:13])
