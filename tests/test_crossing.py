"""Azimuth-crossing dumps (PositionDumpBunch, src/FFAG_dump.py:789-1130).

The golden fixture holds the files the reference wrote for Boris and RK4
loops with crossing dumps registered (tests/golden/make_golden.py
--crossing).  The oracle's step-by-step crossing records, turned into rows
by the product's host code, reproduce them; the GPU loop writes the same
files through ffa_push_crossing."""
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from pyffa_b200.dump import Dumps, PositionDumpBunch
from pyffa_b200.track import crossing_rows

from .fixtures import HERE, load_golden

CROSSING = os.path.join(HERE, "golden", "golden_crossing.npz")
CASES = {"xb": "Boris", "xr": "RK4"}


@pytest.fixture(scope="module")
def xg():
    z = np.load(CROSSING)
    return {k: z[k] for k in z.files}


def _dumps(windows, root):
    return [PositionDumpBunch(deg, t0, t1, save_folder=os.path.join(root, f"d{k}"))
            for k, (deg, t0, t1) in enumerate(windows)]


def _written(d):
    files = sorted(os.listdir(d.save_folder))
    assert len(files) <= 1
    return (files[0], np.load(os.path.join(d.save_folder, files[0]))["particles"]) if files else (None, None)


def _check_dump(got_name, got, xg, key, k, rtol):
    fk = f"{key}_file{k}"
    if fk not in xg:
        assert got_name is None, got_name
        return
    assert got_name == bytes(xg[fk]).decode()
    ref = xg[f"{key}_dump{k}"]
    assert got.shape == ref.shape, (got.shape, ref.shape)
    if rtol == 0:
        assert np.array_equal(got, ref)
        return
    # same particles, same steps (time column), same order
    assert np.array_equal(got[:, 13:16], ref[:, 13:16]) and np.array_equal(got[:, 16], ref[:, 16])
    assert np.array_equal(got[:, [6, 7, 8]], ref[:, [6, 7, 8]])
    for c in (0, 1, 2, 3, 4, 5, 9):
        scale = max(np.abs(ref[:, c]).max(), 1e-300)
        assert np.abs(got[:, c] - ref[:, c]).max() <= rtol * scale, (key, k, c)


def test_detect_crossing_rule():
    tw = 2 * np.pi
    pre = np.array([0.1, 0.1, 6.2, 6.2, 6.2, 0.5, 0.5, 1.0, 3.0, -0.1])
    post = np.array([0.3, 0.3, 6.3, 0.05, 0.05, 0.5, 0.5, 1.2, 3.1, 0.05])
    surv = np.array([1, 0, 1, 1, 1, 1, 1, 1, 1, 1])
    tgt = np.array([0.2, 0.2, 6.25, 6.25, 0.02, 0.5, 0.5, 1.2, 2.0, 0.0])
    got = [O.detect_azimuth_crossing(pre[i:i + 1], post[i:i + 1], surv[i:i + 1], tgt[i]) for i in range(len(pre))]
    hit = [bool(g[0][0]) for g in got]
    ratio = [float(g[1][0]) for g in got]
    assert hit == [True, False, True, True, True, True, True, True, False, True]
    assert ratio[0] == pytest.approx(0.5)
    assert ratio[2] == pytest.approx(0.5)          # 6.3 wraps to 0.0168: crossing through 2 pi
    assert ratio[4] == pytest.approx((0.02 + tw - 6.2) / (0.05 + tw - 6.2))
    assert ratio[5] == 0.0                         # zero span: crossed, ratio 0
    assert ratio[7] == pytest.approx(1.0)


@pytest.mark.parametrize("key", list(CASES))
def test_oracle_crossing_dumps_match_reference(xg, key):
    g = load_golden()
    solver = CASES[key]
    setup = O.Setup(g.bmap(), g.emap(), g.gp(aperture=(solver == "Boris")))
    ts, dt, n = xg[key + "_t"]
    m = xg[key + "_in"].copy()
    windows = xg[key + "_windows"]
    targets = [np.deg2rad(w[0]) % (2 * np.pi) for w in windows]
    rec, _, _ = O.track_crossings(setup, solver, m, ts, dt, int(n), targets)
    tpost = ts + dt * (np.arange(int(n)) + 1)
    t = ts
    for s in range(int(n)):                     # the loop's time by repeated addition
        t = t + dt
        tpost[s] = t
    root = tempfile.mkdtemp()
    for k, d in enumerate(_dumps(windows, root)):
        r = rec[rec[:, 0] == k]
        tp = tpost[r[:, 2].astype(np.int64)]
        keep = d.in_window(tp)
        d.add_particles(crossing_rows(r[keep], xg[key + "_in"]), tp[keep])
        if (tpost > d.end_time).any():
            d.save_all_particles(solver)
        _check_dump(*_written(d), xg, key, k, 0)     # bit-exact
    np.testing.assert_allclose(m[:, :6], xg[key + "_out"][:, :6], rtol=1e-13, atol=1e-15)


def test_position_dump_refuses_nonempty_folder():
    root = tempfile.mkdtemp()
    with open(os.path.join(root, "x"), "w") as f:
        f.write("x")
    with pytest.raises(SystemExit):
        PositionDumpBunch(10.0, 0.0, 1.0, save_folder=root)


@pytest.mark.gpu
@pytest.mark.parametrize("key,precision", [("xb", "fp64"), ("xr", "fp64"), ("xb", "fp32c")])
def test_gpu_crossing_dumps_match_reference(xg, key, precision):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.track import FFAG_RungeKutta
    g = load_golden()
    solver = CASES[key]
    ts, dt, n = xg[key + "_t"]
    gp = g.gp(aperture=(solver == "Boris"))
    b = FFAG_Bunch(xg[key + "_in"].copy(), BunchType=solver)
    root = tempfile.mkdtemp()
    dl = _dumps(xg[key + "_windows"], root)
    dumps = Dumps()
    for d in dl:
        dumps.add_dump(d)
    lp = {"stop_condition": {"max_stepsN": int(n), "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": dumps}
    rk = FFAG_RungeKutta(precision=precision, verbose=False)
    (rk.rk4_solve_dt_bunch3_withSC_boris if solver == "Boris" else rk.rk4_solve_dt_bunch3_withSC)(
        None, ts, b, gp, lp)
    # float64 pushers: the parity tolerance of the loops; fp32c: its float32 increments
    rtol = 1e-11 if precision == "fp64" else 2e-6
    for k, d in enumerate(dl):
        _check_dump(*_written(d), xg, key, k, rtol)
