"""The learned sector map on the time-domain plain pusher: sector maps of the
compensated float32 Boris pusher (TimeDomainSectorTracker: one push launch,
the crossing of the next sector entrance captured and interpolated) generate
the training crossings, audit the network and take over its failures, and
the FP64 Boris pusher at the same step is the reference of the accuracy
figures.

Checks: the time-domain sector map against the azimuth-domain RK4 map (the
same field; the difference is the Boris step's truncation), FP32C against
FP64 at the same step (the float32 field), two sectors against one sector
twice (the interpolation), and the map learned from FP32C crossings over
1000 turns against FP64 Boris: tune error <= 1e-4 and emittance error
<= 1 %, and the network beats its skip connection alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


@pytest.fixture(scope="module")
def td():
    from pyffa_b200 import learned, synthetic
    from pyffa_b200.constants import FFAG_ConversionTools, FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical
    cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=0, AddNumricalMap=False)
    bm.UpdataConfig()
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    dt = synthetic.design_dt(300.0, 2880)
    t32 = learned.TimeDomainSectorTracker(gp, dt, "fp32c")
    t64 = learned.TimeDomainSectorTracker(gp, dt, "fp64")
    rk4 = learned.SectorTracker(gp.Bmap, gp.q, steps_per_sector=256)
    d0 = synthetic.design(300.0)
    conv = FFAG_ConversionTools()
    P = conv.Ek2P(np.cos(np.pi * (np.arange(17) + 0.5) / 17)[::-1] * 150.0 + 450.0)
    r_guess = d0["r0"] * (P / conv.Ek2P(300.0)) ** (1 / (cfg["Bmap"]["coefficients_tupel"][1] + 1))
    frame = learned.SectorFrame.build(t64, (300.0, 600.0), (10e-3, 5e-3), r_guess=r_guess, pr_guess=d0["pr0"])
    return {"frame": frame, "t32": t32, "t64": t64, "rk4": rk4}


def _states(frame, n, seed):
    from pyffa_b200 import learned
    s = torch.from_numpy(learned.sample_domain(n, np.random.default_rng(seed))).cuda()
    P = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(s[:, 4].cpu().numpy())), device="cuda")
    return torch.cat([frame.to_phys(s, s[:, 4]), P[:, None]], 1)


def test_time_domain_sector_map(td):
    frame = td["frame"]
    x = _states(frame, 4096, 1)
    a64 = td["t64"].run(x, 1)
    a32 = td["t32"].run(x, 1)
    b = td["rk4"].run(x, 1)
    # Boris at 240 steps per sector against RK4 at 256: the Boris truncation
    # (the closed orbits of the two differ by ~13 um)
    d = (a64 - b).abs().max(0).values.tolist()
    assert d[0] < 1e-4 and d[2] < 1e-4 and d[1] < 1e-4 and d[3] < 1e-4, d
    # FP32C against FP64 at the same step: the float32 field
    d = (a32 - a64).abs().max(0).values.tolist()
    assert max(d) < 5e-7, d
    # two sectors at once against one sector twice: the second push starts
    # its steps at the interpolated crossing, so the two differ by the Boris
    # truncation at shifted step boundaries, not by a step (~1 cm)
    two = td["t64"].run(x, 2)
    twice = td["t64"].run(torch.cat([a64, x[:, 4:5]], 1), 1)
    d = (two - twice).abs().max(0).values.tolist()
    assert max(d) < 2e-5, d


def test_learned_map_on_fp32c_crossings(td):
    from pyffa_b200 import learned
    frame, t32, t64 = td["frame"], td["t32"], td["t64"]
    X, T = learned.make_dataset(frame, t32, 1 << 22, seed=1)
    Xv, Tv = learned.make_dataset(frame, t32, 1 << 16, seed=2)
    p = torch.from_numpy(learned.init_params(3)).cuda()
    learned.train(p, X, T, epochs=40, batch=8192, lr=2e-3, log_every=0)
    mse = learned.evaluate(p, Xv, Tv)
    quad = p.clone()
    for k in ("W4", "b4"):
        learned.block(quad, k).zero_()
    mse_quad = learned.evaluate(quad, Xv, Tv)
    assert mse < mse_quad / 100, (mse, mse_quad)
    rng = np.random.default_rng(4)
    n, turns = 512, 1000
    s = np.zeros((n, 5))
    s[:, :4] = 0.3 * rng.standard_normal((n, 4))
    for j in (0, 2):
        r = np.hypot(s[:, j], s[:, j + 1])
        s[:, j:j + 2] *= np.minimum(1.0, 0.9 / np.maximum(r, 1e-12))[:, None]
    s[:, 4] = rng.uniform(-0.9, 0.9, n)
    st = torch.from_numpy(s).cuda()
    P = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(s[:, 4])), device="cuda")
    phys = torch.cat([frame.to_phys(st, st[:, 4]), P[:, None]], 1)
    ref = learned.plain_track(frame, t64, phys, turns, record=True)
    out = {}
    for name, prm in (("learned", p), ("second-order", quad)):
        lm = learned.LearnedSectorMap(frame, t32, prm, audit_every=50, audit_frac=0.01, audit_tol=1e-5)
        r = lm.track(phys, turns, record=True)
        dq = np.abs(learned.tunes(r["record"]) - learned.tunes(ref["record"]))
        de = np.abs(learned.betatron_emittance(frame, r["record"][-1]) /
                    learned.betatron_emittance(frame, ref["record"][-1]) - 1).max()
        out[name] = (float(dq.max()), float(de), int(r["plain"].sum()))
    print("\nlearned on FP32C crossings vs FP64 Boris (max dq, emittance error, plain states):", out, mse, mse_quad)
    assert out["learned"][0] <= 1e-4 and out["learned"][1] <= 1e-2, out
    assert out["learned"][0] < out["second-order"][0] / 5, out
