"""Launch shapes of the Boris pushers on the GPU: the block size gives
bit-identical states and crossing records (the same kernel); a register cap
gives the same results to rounding (the code generator may place its
multiply-add fusions differently under a tight cap); the runtime's
occupancy figures follow the caps; and the autotuner times every candidate
on a scan bunch, flags the ones whose results are not bit-identical to the
default shape's and chooses among the others."""
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


def _scan(rf_on, autotune=False):
    from pyffa_b200 import coscan, synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    cfg = synthetic.lattice_bmap(r_range=(7.9, 9.3, 0.002), theta_step_deg=0.02)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2))
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=rf_on)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    d = synthetic.design(300.0)
    E = np.array([300.0, 400.0, 500.0, 600.0])
    k = cfg["Bmap"]["coefficients_tupel"][1]
    scale = (synthetic.momentum(E) / synthetic.momentum(300.0)) ** (1 / (k + 1))
    return gp, coscan.BatchedOrbitScan(gp, E, [700, 1500, 2500, 1300], d["r0"] * scale,
                                       np.full(4, np.arctan(d["pr0"])), d["perimeter"] * scale, sigma=2e-3,
                                       turns=2, seed=5, steps_per_turn=2880, autotune=autotune, tune_steps=300)


def _run(gp, v, dt, precision, shape, nsteps=2500):
    from pyffa_b200.track import CrossingCapture, Pusher, StepClock, _EphemeralBunch
    dev = torch.device("cuda", 0)
    b = _EphemeralBunch(v, "Boris", dev)
    p = Pusher(b, gp, "Boris", precision)
    p.shape = shape
    clock = StepClock(0.0, dt, gp.Emap, "Boris", dev)
    clock.ensure(nsteps + 1)
    cap = CrossingCapture(b, [0.0], gp, dt)
    x = cap.prepare(nsteps)
    p.push(clock, 0, nsteps, 0, xing=x)
    torch.cuda.synchronize()
    state = torch.stack([b.cols[k] for k in ("r", "vr", "z", "vz", "fi", "f5", "rf")]).cpu().numpy()
    surv = b.cols["surv"].cpu().numpy()
    return state, surv, cap.records()


@pytest.mark.parametrize("precision,rf_on", [("fp32c", False), ("fp64", True)])
def test_every_shape_gives_identical_results(precision, rf_on):
    from pyffa_b200 import autotune
    gp, scan = _scan(rf_on)
    v = scan._vformat()
    ref = None
    shapes = autotune.candidates(fp32c=precision == "fp32c")
    assert len(shapes) == (16 if precision == "fp32c" else 4)
    report = {}
    for shape in shapes:
        out = _run(gp, v, scan.dt, precision, shape)
        assert out[2].shape[0] > 0 and np.isfinite(out[0]).all()
        if ref is None:
            ref = out
            continue
        same = np.array_equal(out[0], ref[0]) and np.array_equal(out[2], ref[2])
        rel = float(np.max(np.abs(out[0] - ref[0]) / np.maximum(np.abs(ref[0]), 1e-30)))
        report[shape] = (same, rel)
        assert np.array_equal(out[1], ref[1]), shape                 # the same particles survive
        assert out[2].shape == ref[2].shape, shape                   # and cross the azimuth as often
        if shape[1] == 0:
            assert same, shape                                       # block size alone: bit-identical
        else:
            assert rel < 1e-9, (shape, rel)                          # a register cap: rounding at most
    print(precision, {f"{t}x{r}": v for (t, r), v in report.items()})


def test_occupancy_follows_register_cap():
    from pyffa_b200 import _lib, autotune
    warps = []
    for r in range(4):
        blocks, tb = autotune.occupancy(_lib.FFA_FP32C | _lib.shape_flags(1, r), 2, True)
        assert tb == 64 and 1 <= blocks <= 32
        warps.append(blocks * tb // 32)
    assert warps == sorted(warps) and warps[0] < warps[-1], warps


def test_autotuner_times_every_candidate():
    from pyffa_b200 import _lib
    gp, scan = _scan(False, autotune=True)
    scan._setup()
    res = scan.tuning
    assert len(res.rows) == 16
    assert all(r["ms"] > 0 and 1 <= r["warps_per_sm"] <= 64 for r in res.rows)
    assert res.best in [r["shape"] for r in res.rows]
    assert scan._dev_state.pusher.shape == res.best
    assert res.best_ms <= res.default_ms
    # block sizes alone are bit-identical; the chosen shape is within the
    # scan's tolerance, and with none only bit-identical shapes are taken
    assert all(r["identical"] for r in res.rows if r["shape"][1] == 0)
    assert all(r["max_rel_diff"] < 1e-9 for r in res.rows)
    assert next(r for r in res.rows if r["shape"] == res.best)["accepted"]
    from pyffa_b200 import autotune
    exact = [dict(r, accepted=r["identical"]) for r in res.rows]
    assert next(r for r in exact if r["shape"] == autotune.select(exact, 0.02))["identical"]
    rep = res.report()
    assert rep["chosen"]["threads"] in _lib.SHAPE_THREADS and rep["chosen"]["max_regs"] in _lib.SHAPE_NREGS
