"""Parity of the CUDA pushers (through libffa_cuda.so) with the reference.

Tolerances: the CUDA and glibc transcendental functions (pow, exp, sin/cos,
atan2) differ by an ulp or so and the CUDA build fuses multiply-adds, so
float64 coordinates are compared at 1e-12 relative per turn of tracking (the
bar of the tracking path).  Flags (injection, aperture loss) and map cell
indices are compared exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from pyffa_b200 import _lib
    _lib.lib()  # fails loudly if the library is missing


# r, fi, dfi/dt (or Etot) and the RF phase never cross zero: compared per
# element; vr, z, vz and the space-charge fields oscillate through zero and are
# compared relative to their column's largest magnitude (the amplitude).
ELEMENTWISE = (0, 4, 5, 9)
AMPLITUDE = (1, 2, 3, 10, 11, 12)


def coord_errors(m, ref):
    errs = {}
    for c in ELEMENTWISE:
        errs[c] = float(np.max(np.abs(m[:, c] - ref[:, c]) / np.maximum(np.abs(ref[:, c]), 1e-300)))
    for c in AMPLITUDE:
        amp = np.abs(ref[:, c]).max()
        errs[c] = float(np.abs(m[:, c] - ref[:, c]).max() / amp) if amp > 0 else float(np.abs(m[:, c]).max())
    return errs


def _assert_close(m, ref, rtol, floor=None):
    """floor: per-column errors of the oracle against itself when its input
    r is perturbed by one ulp -- the rounding sensitivity of the dynamics over
    the same steps.  The GPU must agree with the oracle to rtol or to ten
    times that floor, whichever is larger."""
    assert np.array_equal(m[:, 7:9], ref[:, 7:9]), "injection / survival flags differ"
    for c, err in coord_errors(m, ref).items():
        tol = max(rtol, 10 * floor[c]) if floor is not None else rtol
        assert err <= tol, f"column {c}: relative error {err:.3g} > {tol:.3g}"


def ulp_floor(S, solver, v, t0, dt, nsteps, ref):
    """Oracle run with r nudged by one ulp, compared with the unperturbed run."""
    from oracle import oracle as O
    pert = v.copy()
    pert[:, 0] = np.nextafter(pert[:, 0], np.inf)
    O.track(S, solver, pert, t0, dt, nsteps)
    return coord_errors(pert, ref)


def test_boris_step_matches_reference_golden(golden):
    from pyffa_b200.track import FFAG_RungeKutta
    t0, dt = golden["boris1_t"]
    m = golden["boris1_in"].copy()
    FFAG_RungeKutta().Boris_solve(t0, m, dt, golden.gp())
    _assert_close(m, golden["boris1_out"], 1e-14)


def test_rk4_step_matches_reference_golden(golden):
    from pyffa_b200.track import FFAG_RungeKutta
    t0, dt = golden["boris1_t"]
    m = golden["rk41_in"].copy()
    dr, *_ = FFAG_RungeKutta().rk4_step_malloc(None, t0, m, dt, golden.gp())
    _assert_close(m + dr, golden["rk41_out"], 1e-14)


@pytest.mark.parametrize("name,solver", [("borisloop", "Boris"), ("rk4loop", "RK4")])
def test_tracking_loop_matches_reference_golden(golden, name, solver):
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.track import FFAG_RungeKutta
    from pyffa_b200.dump import Dumps
    ts, dt, n = golden[name + "_t"]
    b = FFAG_Bunch(golden[name + "_in"], BunchType=solver)
    lp = {"stop_condition": {"max_stepsN": int(n), "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
    rk = FFAG_RungeKutta(verbose=False)
    getattr(rk, "rk4_solve_dt_bunch3_withSC_boris" if solver == "Boris" else "rk4_solve_dt_bunch3_withSC")(
        None, ts, b, golden.gp(), lp)
    _assert_close(b.LocalBunch, golden[name + "_out"], 1e-12)


@pytest.fixture(scope="module")
def full_lattice():
    """The 12-sector lattice on the full 1301 x 6000 map with z-Taylor order 2."""
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    import os
    import tempfile
    cfg = synthetic.lattice_bmap()
    stacks = synthetic.taylor_stacks(cfg, 2)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=stacks)
    d = tempfile.mkdtemp()
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(d, "emap.txt")), EnableFlag=True)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    gp.AddAperture(7.5, 9.5, -0.1, 0.1)
    return gp


@pytest.mark.parametrize("solver,turns", [("Boris", 2), ("RK4", 1)])
def test_full_map_turns_vs_oracle(full_lattice, solver, turns):
    """A seeded 6D Gaussian bunch, RF on (reference last-gap semantics), full
    1301 x 6000 map: per-particle agreement after whole turns."""
    from oracle import oracle as O
    from pyffa_b200 import synthetic
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.constants import FFAG_ConversionTools
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    gp = full_lattice
    n = 512
    p = synthetic.centred_bunch(n, seed=3)
    conv = FFAG_ConversionTools()
    v = conv.ConvertPrzek2Vrzek_boris(p) if solver == "Boris" else conv.ConvertPrzek2Vrzek(p)
    v[:, 9] = 0.7
    dt = synthetic.design_dt(300.0, 720)
    nsteps = 720 * turns
    v_in = v.copy()
    ref = v.copy()
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    O.track(S, solver, ref, 0.0, dt, nsteps)
    b = FFAG_Bunch(v_in, BunchType=solver)
    lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
    rk = FFAG_RungeKutta(verbose=False)
    getattr(rk, "rk4_solve_dt_bunch3_withSC_boris" if solver == "Boris" else "rk4_solve_dt_bunch3_withSC")(
        None, 0.0, b, gp, lp)
    got = b.LocalBunch
    assert (got[:, 8] == 1).sum() > n // 2
    _assert_close(got, ref, 1e-12 * turns, ulp_floor(S, solver, v, 0.0, dt, nsteps, ref))


def test_subset_parity_at_full_size(full_lattice):
    """Particles are independent, so parity on a subset of a 1e5-particle
    bunch pushed as a whole (the benchmark's size) is parity of the whole."""
    from oracle import oracle as O
    from pyffa_b200 import synthetic
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.constants import FFAG_ConversionTools
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    gp = full_lattice
    n = 100_000
    p = synthetic.centred_bunch(n, seed=7)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    dt = synthetic.design_dt(300.0, 720)
    b = FFAG_Bunch(v, BunchType="Boris")
    lp = {"stop_condition": {"max_stepsN": 720, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
    FFAG_RungeKutta(verbose=False).rk4_solve_dt_bunch3_withSC_boris(None, 0.0, b, gp, lp)
    got = b.LocalBunch
    idx = np.random.Generator(np.random.PCG64(0)).choice(n, 400, replace=False)
    idx.sort()
    ref = v[idx].copy()
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    O.track(S, "Boris", ref, 0.0, dt, 720)
    _assert_close(got[idx], ref, 1e-12, ulp_floor(S, "Boris", v[idx], 0.0, dt, 720, ref))
    # whole-bunch properties: nothing non-finite, every particle advanced ~one turn
    assert np.isfinite(got[:, :6]).all()
    alive = got[:, 8] == 1
    turns = got[alive, 4] / (2 * np.pi)
    assert np.all(np.abs(turns - 1.0) < 0.05)


def test_status_counts_losses(golden):
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.dump import Dumps
    from pyffa_b200.track import FFAG_RungeKutta
    ts, dt, n = golden["borisloop_t"]
    b = FFAG_Bunch(golden["borisloop_in"], BunchType="Boris")
    lp = {"stop_condition": {"max_stepsN": int(n), "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
    rk = FFAG_RungeKutta(verbose=False)
    rk.rk4_solve_dt_bunch3_withSC_boris(None, ts, b, golden.gp(), lp)
    ref = golden["borisloop_out"]
    assert rk.last_run["status"]["lost"] == int(((ref[:, 7] == 1) & (ref[:, 8] == 0)).sum())
    assert rk.last_run["status"]["nan"] == 0


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_host_matrix_entry_point_matches_device_push(full_lattice, precision):
    """MatrixTracker (host matrix in, one call, host matrix out) gives the
    device push's result bit for bit, with one stream and with the bunch
    split over two streams (copies of one half overlapping the other's
    push); a ragged size exercises the split at a multiple of 32."""
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    from pyffa_b200.track import MatrixTracker, Pusher, StepClock, _EphemeralBunch
    gp = full_lattice
    n = 3001
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(synthetic.centred_bunch(n, seed=11))
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    v[:, 9] = 0.3
    dt = synthetic.design_dt(300.0, 720)
    dev = torch.device("cuda", 0)
    b = _EphemeralBunch(v.copy(), "Boris", dev)
    pu = Pusher(b, gp, "Boris", precision)
    clock = StepClock(0.0, dt, gp.Emap, "Boris", dev)
    clock.ensure(2 * 720)
    pu.push(clock, 0, 720, 0)
    pu.push(clock, 720, 720, 0)
    torch.cuda.synchronize()
    ref = b.matrix()
    for chunks in (1, 2):
        mt = MatrixTracker(n, gp, "Boris", precision, device=dev, chunks=chunks)
        mt.bind_clock(0.0, dt, 2 * 720)
        assert len(mt.spans) == chunks and all(a % 32 == 0 for a, _ in mt.spans)
        h = [torch.from_numpy(v.copy()).pin_memory(), torch.zeros((n, 16), dtype=torch.float64).pin_memory()]
        mt.run(h[0], h[1], 0, 720)
        mt.run(h[1], h[0], 720, 720)
        mt.pusher.stream.synchronize()
        got = h[0].numpy()
        cols = [0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11, 12]
        assert np.array_equal(got[:, cols], ref[:, cols]), chunks
        assert int(mt.b.status[_lib_status_lost()].item()) == int(b.status[_lib_status_lost()].item())


def _lib_status_lost():
    from pyffa_b200 import _lib
    return _lib.STATUS_LOST


def test_c0_hundred_turns_vs_oracle():
    """Workload c0: plain float64 Boris, no RF, no space charge, the full
    1301 x 6000 map with z-Taylor order 2, a 1e4-particle seeded 6D Gaussian
    bunch, 100 turns of 720 steps.  The whole bunch is pushed on the GPU one
    turn per launch; after every turn a 512-particle subset is compared with
    the oracle's run of the same particles, per element, at 1e-12 per turn or
    ten times the dynamics' own rounding sensitivity over the same turns,
    whichever is larger.  That sensitivity is the largest of three measures:
    the oracle against itself with r nudged by one ulp; the oracle against its
    build with fused multiply-adds (a second correct float64 build that rounds
    differently at every contracted operation); and the oracle against its run
    with every state value's last bit flipped or kept at random after every
    step (orc_track_noisy: rounding differences at every step, as between the
    GPU's math functions and the host's).  At 720 steps per turn the
    large-amplitude motion is weakly chaotic, so the sensitivity itself grows
    from 1e-14 to ~1e-7 of the vertical amplitude over the run; the noise
    measure runs 4-6x above the fused build's.  Loss flags are exact while the
    oracle's own runs agree on them; later, a particle that grazes the
    aperture may be lost a turn earlier or later (rules in the loop)."""
    import os
    import tempfile
    from oracle import oracle as O
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools, FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    from pyffa_b200.track import Pusher, StepClock, _EphemeralBunch
    cfg = synthetic.lattice_bmap()
    gp = FFAG_GlobalParameters()
    gp.AddBMap(FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2)))
    gp.AddEMap(FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=False))
    gp.AddAperture(7.5, 9.5, -0.1, 0.1)
    n, turns, spt = 10_000, 100, 720
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(synthetic.centred_bunch(n, seed=5))
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    dt = synthetic.design_dt(300.0, spt)
    idx = np.sort(np.random.Generator(np.random.PCG64(1)).choice(n, 512, replace=False))
    dev = torch.device("cuda", 0)
    b = _EphemeralBunch(v.copy(), "Boris", dev)
    pu = Pusher(b, gp, "Boris", "fp64")
    clock = StepClock(0.0, dt, gp.Emap, "Boris", dev)
    clock.ensure(turns * spt)
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    ref = v[idx].copy()
    nudged = ref.copy()
    nudged[:, 0] = np.nextafter(nudged[:, 0], np.inf)
    fused = ref.copy()
    noisy = ref.copy()
    worst = []
    split = np.zeros(len(idx), bool)       # particles whose loss turn differs between any two runs
    for t in range(1, turns + 1):
        pu.push(clock, (t - 1) * spt, spt, 0)
        torch.cuda.synchronize()
        got = b.matrix()[idx]
        O.track(S, "Boris", ref, clock.t[(t - 1) * spt], dt, spt)
        O.track(S, "Boris", nudged, clock.t[(t - 1) * spt], dt, spt)
        O.track(S, "Boris", fused, clock.t[(t - 1) * spt], dt, spt, fused=True)
        O.track(S, "Boris", noisy, clock.t[(t - 1) * spt], dt, spt, noise=(1, (t - 1) * spt))
        # loss flags: a particle that grazes the aperture is lost a turn
        # earlier or later under rounding changes once the motion has
        # diverged; the GPU may split from the oracle on no more particles
        # than the oracle splits from itself (twice the largest of the three
        # measures), and on one after turn 50; split particles leave the
        # coordinate comparison
        def flag_split(m):
            return np.any(m[:, 7:9] != ref[:, 7:9], axis=1)
        s_own = [flag_split(m) for m in (nudged, fused, noisy)]
        s_gpu = flag_split(got)
        allowed = 2 * max(int(x.sum()) for x in s_own) + (1 if t > 50 else 0)
        assert int(s_gpu.sum()) <= allowed, f"flags differ after turn {t} on {int(s_gpu.sum())} particles"
        split |= s_gpu
        for x in s_own:
            split |= x
        keep = ~split
        fn, ff, fr = (coord_errors(m[keep], ref[keep]) for m in (nudged, fused, noisy))
        floor = {c: max(fn[c], ff[c], fr[c]) for c in fn}
        errs = coord_errors(got[keep], ref[keep])
        for c, err in errs.items():
            tol = max(1e-12 * t, 10 * floor[c])
            assert err <= tol, f"turn {t}, column {c}: relative error {err:.3g} > {tol:.3g}"
        worst.append(max(errs[c] for c in ELEMENTWISE))
    assert (ref[:, 8] == 1).sum() > 256 and split.sum() < 16, int(split.sum())
    print("\nc0: largest per-element error of r, fi, dfi/dt, RF phase after turns 1, 10, 100:",
          worst[0], worst[9], worst[-1])
