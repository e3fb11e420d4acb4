"""Batched orbit scan on the GPU: five instances (1 to 120 particles,
300-600 MeV) through the compensated float32 pusher in one bunch; the
fitted closed orbits agree with the scaling-law orbit of the azimuth-domain
search and the fractional tunes with its one-sector transfer matrix, and a
second iteration (a replay of the iteration's CUDA graph) changes the
orbits by less than the first."""
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


def test_batched_scan_orbits_and_tunes():
    from pyffa_b200 import coscan, synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    cfg = synthetic.lattice_bmap(r_range=(7.9, 9.3, 0.002), theta_step_deg=0.02)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2))
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=False)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    d = synthetic.design(300.0)
    E = np.array([300.0, 375.0, 450.0, 525.0, 600.0])
    k = cfg["Bmap"]["coefficients_tupel"][1]
    scale = (synthetic.momentum(E) / synthetic.momentum(300.0)) ** (1 / (k + 1))
    r_exp = d["r0"] * scale
    pr_exp = np.full(len(E), np.arctan(d["pr0"]))
    # start 0.2 mm off the orbit
    counts = [1, 4, 30, 120, 9]
    scan = coscan.BatchedOrbitScan(gp, E, counts, r_exp + 2e-4, pr_exp, d["perimeter"] * scale,
                                   sigma=0.5e-3, turns=60, seed=3, steps_per_turn=2880)
    first = scan.iterate()
    second = scan.iterate()           # the captured CUDA graph of an iteration, replayed
    assert (first["mode"], second["mode"]) == ("captured", "graph")
    assert first["good"].all() and second["good"].all()
    # the first update takes the orbit most of the way, the second is small
    assert first["max_abs_dr"] > 1e-4 and second["max_abs_dr"] < 2e-5, (first["max_abs_dr"], second["max_abs_dr"])
    # the time-domain orbit (Boris, 2880-3330 steps per turn) is the azimuth-domain one to discretisation error
    assert np.abs(scan.r - r_exp).max() < 1e-4, scan.r - r_exp
    assert np.abs(scan.z).max() < 1e-6
    q = second["tunes"]
    assert np.abs(q[:, 0] - (d["Qx"] % 1)).max() < 2e-3, q
    assert np.abs(q[:, 1] - (d["Qz"] % 1)).max() < 2e-3, q
    # every particle crossed the azimuth at least once per turn of the slowest instance
    assert (second["crossings"] >= 60 * np.array(counts)).all()
    # self-consistency: 10 um offsets around the orbit found come back to it
    check = coscan.BatchedOrbitScan(gp, E, [8] * 5, scan.r, scan.pr, d["perimeter"] * scale,
                                    sigma=1e-5, turns=60, seed=4, steps_per_turn=2880)
    rec = check.iterate(graph=False)  # the direct path, no graph
    assert rec["mode"] == "direct"
    assert rec["good"].all() and rec["max_abs_dr"] < 3e-6, rec["max_abs_dr"]


def test_one_launch_and_many_launches_agree():
    """With crossing records: the persistent iteration (one push launch, all records in one buffer)
    and the same iteration in launches of at most 5 records per particle give
    the same orbit update (to rounding: a launch boundary re-forms 1 / r)."""
    from pyffa_b200 import coscan, synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    cfg = synthetic.lattice_bmap(r_range=(7.9, 9.3, 0.002), theta_step_deg=0.02)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2))
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=False)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    d = synthetic.design(300.0)
    E = np.array([300.0, 450.0, 600.0])
    k = cfg["Bmap"]["coefficients_tupel"][1]
    scale = (synthetic.momentum(E) / synthetic.momentum(300.0)) ** (1 / (k + 1))
    out = []
    for persistent in (True, False):
        scan = coscan.BatchedOrbitScan(gp, E, [16, 40, 9], d["r0"] * scale + 2e-4, np.full(3, np.arctan(d["pr0"])),
                                       d["perimeter"] * scale, sigma=0.5e-3, turns=20, seed=6, steps_per_turn=2880,
                                       autotune=False, persistent=persistent, accumulate="records")
        rec = scan.iterate(graph=False)
        out.append((rec, scan.r.copy(), scan._dev_state.launches))
    (a, ra, la), (b, rb, lb) = out
    assert la == 1 and lb > 1, (la, lb)
    assert np.array_equal(a["crossings"], b["crossings"])
    assert np.abs(ra - rb).max() < 1e-9, ra - rb
    assert np.abs(a["tunes"] - b["tunes"]).max() < 1e-7


def test_kernel_sums_equal_record_sums():
    """The normal equations the push kernel accumulates at crossing time
    (ffa_crossing.fit_sums) against the same iteration with crossing records
    reduced by accumulate_crossings_fixed: the pushes are the same kernel
    and launch, so the particles' states are identical and the sums differ
    by the interpolation's rounding (the kernel reduces the azimuth mod 2 pi
    before its sine and cosine) and the order of the float64 atomics."""
    from pyffa_b200 import coscan, synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    cfg = synthetic.lattice_bmap(r_range=(7.9, 9.3, 0.002), theta_step_deg=0.02)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2))
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=False)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    d = synthetic.design(300.0)
    E = np.array([300.0, 420.0, 510.0, 600.0])
    k = cfg["Bmap"]["coefficients_tupel"][1]
    scale = (synthetic.momentum(E) / synthetic.momentum(300.0)) ** (1 / (k + 1))
    counts = [1, 33, 200, 7]
    out = {}
    for mode in ("kernel", "records"):
        scan = coscan.BatchedOrbitScan(gp, E, counts, d["r0"] * scale + 2e-4, np.full(4, np.arctan(d["pr0"])),
                                       d["perimeter"] * scale, sigma=0.5e-3, turns=25, seed=8, steps_per_turn=2880,
                                       autotune=False, accumulate=mode)
        rec = scan.iterate(graph=False)
        st = scan._dev_state
        assert st.launches == 1
        if mode == "kernel":
            S, Y, c = coscan.unpack_fit_sums(st.sums.cpu().numpy())
            assert not hasattr(st, "rows")          # no record buffer
        else:
            S, Y = st.S[:, :4].cpu().numpy(), st.Y[:, :4].cpu().numpy()
            c = st.crossings[:4].cpu().numpy()
        out[mode] = (S, Y, c, rec, scan.r.copy(), scan.pr.copy())
    (Sk, Yk, ck, rk, rrk, prk), (Sr, Yr, cr, rr, rrr, prr) = out["kernel"], out["records"]
    np.testing.assert_array_equal(ck, cr)
    assert (ck >= 25 * np.array(counts)).all()
    for A, B in ((Sk, Sr), (Yk, Yr)):
        scale_ = np.abs(B).max(axis=(2, 3), keepdims=True)
        assert (np.abs(A - B) <= 1e-10 * scale_).all(), np.abs(A - B).max()
    assert np.abs(rrk - rrr).max() < 1e-11, rrk - rrr
    assert np.abs(prk - prr).max() < 1e-11
    assert np.nanmax(np.abs(rk["tunes"] - rr["tunes"])) < 1e-9
    np.testing.assert_array_equal(rk["good"], rr["good"])
