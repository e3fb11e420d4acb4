"""Learned sector map on the GPU: the tensor-core GEMM, the training step's
loss, gradients and Adam update, and the fused inference kernel, each
against the CPU oracle network (oracle/mlp.py) on the same seeded inputs;
then the whole method on the lattice: train on crossings of the plain
tracker, track 1000 turns, and compare tunes and emittances with the FP64
plain tracker — and with the linear map alone (the method without the
network)."""
import ctypes

import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _params(seed, scale_out=0.05):
    from pyffa_b200 import learned
    rng = np.random.default_rng(seed)
    d = learned.to_dict(learned.init_params(seed))
    d["W4"] = rng.standard_normal(d["W4"].shape) * scale_out / 16
    for k in ("b1", "b2", "b3"):
        d[k] = 0.1 * rng.standard_normal(d[k].shape)
    d["b4"] = 0.01 * rng.standard_normal(6)
    d["Ws"] = 0.1 * rng.standard_normal((6, 6))
    d["bs"] = 0.01 * rng.standard_normal(6)
    d["Wq"] = 0.05 * rng.standard_normal((15, 6))
    return {k: v.astype(np.float32).astype(np.float64) for k, v in d.items()}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("tA,tB", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("Mm,Nn,Kk", [(100, 72, 40),        # narrow: the mma.sync kernel
                                      (300, 260, 200),      # tcgen05, ragged tiles and K
                                      (512, 256, 1024)])    # tcgen05, full tiles
def test_gemm_matches_bf16_products(tA, tB, Mm, Nn, Kk):
    import ctypes
    from pyffa_b200 import _lib
    rng = np.random.default_rng(10 + 2 * tA + tB + Mm)
    A = rng.standard_normal((Kk, Mm) if tA else (Mm, Kk)).astype(np.float32)
    B = rng.standard_normal((Nn, Kk) if tB else (Kk, Nn)).astype(np.float32)
    bias = rng.standard_normal(Nn).astype(np.float32)
    dA, dB, db = (torch.from_numpy(v).cuda() for v in (A, B, bias))
    C = torch.full((Mm, Nn), float("nan"), device="cuda")
    rc = _lib.lib().ffa_mlp_gemm(dA.data_ptr(), A.shape[1], tA, dB.data_ptr(), B.shape[1], tB, C.data_ptr(), Nn,
                                 Mm, Nn, Kk, db.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    opA = M.bf16(A).T if tA else M.bf16(A)
    opB = M.bf16(B).T if tB else M.bf16(B)
    ref = opA @ opB + bias
    got = C.cpu().numpy()
    assert np.all(np.isfinite(got))
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    cnt = ctypes.c_int32(-1)
    assert _lib.lib().ffa_mlp_gemm_timeouts(ctypes.byref(cnt)) == 0 and cnt.value == 0


def _train_inputs(seed, B):
    rng = np.random.default_rng(seed)
    x = np.zeros((B, 8), np.float32)
    x[:, :5] = rng.uniform(-1, 1, (B, 5))
    t = np.zeros((B, 8), np.float32)
    t[:, :5] = x[:, :5] + 0.05 * rng.standard_normal((B, 5))
    return x, t


@pytest.mark.parametrize("B", [512, 1000])
def test_train_step_gradients_match_oracle(B):
    from pyffa_b200 import learned
    d = _params(20)
    p = torch.from_numpy(learned.from_dict(d)).cuda()
    x, t = _train_inputs(21, B)
    tr = learned.Trainer(p, batch=B, n_fit=4, freeze_skip=False)
    tr.step(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), 0.0)
    torch.cuda.synchronize()
    g = learned.to_dict(tr.g.cpu().numpy())
    x6, t6 = x[:, :6].astype(np.float64), t[:, :6].astype(np.float64)
    sse16, g16 = M.loss_and_grads(d, x6, t6, n_fit=4, bf16_ops=True)
    sse64, g64 = M.loss_and_grads(d, x6, t6, n_fit=4)
    # the kernels evaluate SiLU as h + h tanh(h) with the hardware tanh
    # approximation (relative error below 2^-10.9), a few 1e-4 of each
    # activation on top of the float32 accumulation of bfloat16 operands
    assert abs(tr.loss_part.sum().item() - sse16) <= 3e-3 * sse16
    for k in g16:
        assert _rel(g[k], g16[k]) <= 1e-2, (k, _rel(g[k], g16[k]))
        # and within bfloat16 rounding of the exact float64 gradient
        assert _rel(g[k], g64[k]) <= 5e-2, (k, _rel(g[k], g64[k]))
    assert not g["W4"][:, 4:].any() and not g["b4"][4:].any()
    # parameters are untouched by an lr = 0 step
    assert np.array_equal(p.cpu().numpy(), learned.from_dict(d))


def test_adam_step_matches_oracle():
    from pyffa_b200 import learned
    d = _params(22)
    p = torch.from_numpy(learned.from_dict(d)).cuda()
    x, t = _train_inputs(23, 512)
    tr = learned.Trainer(p, batch=512, n_fit=4, freeze_skip=True)
    xs, ts = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    ref = {k: v.copy() for k, v in d.items()}
    m = {k: np.zeros_like(v) for k, v in d.items()}
    v = {k: np.zeros_like(v) for k, v in d.items()}
    for step in (1, 2, 3):
        tr.step(xs, ts, 1e-3)
        torch.cuda.synchronize()
        g = learned.to_dict(tr.g.cpu().numpy())     # the step's own gradients
        M.adam(ref, g, m, v, step, 1e-3, frozen=("Ws", "bs", "Wq"))
        got = learned.to_dict(p.cpu().numpy())
        for k in ref:
            assert np.abs(got[k] - ref[k]).max() <= 1e-6 * max(1.0, np.abs(ref[k]).max()), (step, k)
    for k in ("Ws", "bs", "Wq"):
        assert np.array_equal(got[k], d[k])


@pytest.mark.parametrize("n,n_apply", [(1000, 1), (333, 3), (40_000, 2)])
def test_inference_matches_oracle(n, n_apply):
    from pyffa_b200 import learned
    d = _params(30, scale_out=0.2)
    p = torch.from_numpy(learned.from_dict(d)).cuda()
    rng = np.random.default_rng(31)
    s = np.zeros((n, 8), np.float32)
    s[:, :5] = rng.uniform(-0.7, 0.7, (n, 5))
    s[::17, 0] = 1.3          # outside the domain from the start
    s[5::23, 4] = -1.2
    lm = learned.LearnedSectorMap(None, None, p, radius=1.0)
    st = torch.from_numpy(s).cuda()
    applied = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    lm.apply(st, n_apply, applied)
    torch.cuda.synchronize()
    ref, ref_app = M.apply_map(d, s[:, :6].astype(np.float64), n_apply, radius2=1.0, bf16_ops=True)
    got = st.cpu().numpy()
    app = applied.cpu().numpy()
    assert np.array_equal(app, ref_app)
    assert np.array_equal(got[:, 4:], s[:, 4:])                   # e and the padding stay
    out = app == 0
    assert np.array_equal(got[out], s[out])
    # bfloat16 operands: the kernel's SiLU (hardware tanh approximation,
    # relative error below 2^-10.9) and float32 accumulation order put an
    # occasional activation on the other side of a bfloat16 rounding boundary
    # from the float64 oracle's (a 2^-8 relative step of that one
    # activation), so the bound is on the distribution of the differences
    diff = np.abs(got[:, :4] - ref[:, :4])
    assert np.median(diff) <= 2e-5 * n_apply, np.median(diff)
    assert np.quantile(diff, 0.99) <= 2e-4 * n_apply, np.quantile(diff, 0.99)
    assert diff.max() <= 2e-3 * n_apply, diff.max()
    assert lm.error_flag() == 0
    # and within bfloat16 rounding of the exact float64 network, where that
    # network takes the same domain decisions (a state that bfloat16 rounding
    # moves across the domain boundary gets one map more or less)
    ref64, app64 = M.apply_map(d, s[:, :6].astype(np.float64), n_apply, radius2=1.0, bf16_ops=False)
    same = app64 == app
    assert same.mean() > 0.999
    assert np.abs(got[same, :4] - ref64[same, :4]).max() <= 2e-2 * n_apply


def test_paired_tiles_match_single_tile_kernel():
    """More 128-state tiles than SMs run two tiles in flight per SM (the
    paired kernel, an unpaired last tile in slot 0 alone); the same states in
    pieces of at most one tile per SM run the single-tile kernel.  Both issue
    the same products in the same order and the same epilogue arithmetic:
    bit-identical states and map counts."""
    from pyffa_b200 import learned
    d = _params(32, scale_out=0.2)
    p = torch.from_numpy(learned.from_dict(d)).cuda()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    n = 128 * (2 * sms + 37) + 45          # pairs, unpaired last tiles, a ragged tile
    rng = np.random.default_rng(33)
    s = np.zeros((n, 8), np.float32)
    s[:, :5] = rng.uniform(-0.7, 0.7, (n, 5))
    s[::17, 0] = 1.3
    s[5::23, 4] = -1.2
    lm = learned.LearnedSectorMap(None, None, p, radius=1.0)
    a = torch.from_numpy(s).cuda()
    b = a.clone()
    app_a = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    app_b = app_a.clone()
    lm.apply(a, 3, app_a)
    step = 128 * sms
    for k in range(0, n, step):
        lm.apply(b[k:k + step], 3, app_b[k:k + step])
    torch.cuda.synchronize()
    assert lm.error_flag() == 0
    assert torch.equal(app_a, app_b) and int((app_a == 3).sum()) > n // 2
    assert torch.equal(a, b)
    assert not torch.equal(a, torch.from_numpy(s).cuda())


@pytest.fixture(scope="module")
def lattice():
    from pyffa_b200 import learned, synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters, FFAG_ConversionTools
    from pyffa_b200.fields import FFAG_Bfield_analytical
    cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=0, AddNumricalMap=False)
    bm.UpdataConfig()
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    tracker = learned.SectorTracker(gp.Bmap, gp.q, steps_per_sector=128)
    d0 = synthetic.design(300.0)
    conv = FFAG_ConversionTools()
    P = conv.Ek2P(np.cos(np.pi * (np.arange(17) + 0.5) / 17)[::-1] * 150.0 + 450.0)
    r_guess = d0["r0"] * (P / conv.Ek2P(300.0)) ** (1 / (cfg["Bmap"]["coefficients_tupel"][1] + 1))
    frame = learned.SectorFrame.build(tracker, (300.0, 600.0), (10e-3, 5e-3), r_guess=r_guess, pr_guess=d0["pr0"])
    return {"frame": frame, "tracker": tracker, "design": d0}


def test_frame_round_trip_and_closed_orbit(lattice):
    from pyffa_b200 import learned
    frame, tracker = lattice["frame"], lattice["tracker"]
    # the design closed orbit at 300 MeV is the frame's origin
    # (the design's pr0 is p_r / p_theta, the tracker's p_r / p)
    r, pr = frame.co(frame.e_of(300.0))
    pr0 = lattice["design"]["pr0"] / np.sqrt(1 + lattice["design"]["pr0"] ** 2)
    assert abs(r - lattice["design"]["r0"]) < 1e-7 and abs(pr - pr0) < 1e-7
    # the tunes of the one-sector matrix are the design tunes (scaling
    # lattice: the same at every energy), to the step size of the trackers
    assert abs(frame.tunes[0] - lattice["design"]["Qx"]) < 1e-4
    assert abs(frame.tunes[1] - lattice["design"]["Qz"]) < 1e-4
    s = torch.from_numpy(learned.sample_domain(1000, np.random.default_rng(1))).cuda()
    ph = frame.to_phys(s, s[:, 4])
    P = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(s[:, 4].cpu().numpy())), device="cuda")
    back = frame.to_norm(torch.cat([ph, P[:, None]], 1))
    assert (back - s).abs().max().item() < 1e-11
    # amplitude 1 reaches at most 10 mm / 5 mrad
    assert (ph[:, 0] - frame.co(s[:, 4])[0]).abs().max().item() <= 10e-3 * (1 + 1e-12)


def test_learned_map_gain_tunes_and_emittance(lattice):
    """Train, then 1000 turns of a bunch: the learned map against the FP64
    plain tracker, and the same skip connection without the network (the
    least-squares second-order map) and the linear map against it."""
    from pyffa_b200 import learned
    frame, tracker = lattice["frame"], lattice["tracker"]
    X, T = learned.make_dataset(frame, tracker, 1 << 22, seed=1)
    Xv, Tv = learned.make_dataset(frame, tracker, 1 << 16, seed=2)
    p = torch.from_numpy(learned.init_params(3)).cuda()
    learned.train(p, X, T, epochs=40, batch=8192, lr=2e-3, log_every=0)
    mse = learned.evaluate(p, Xv, Tv)
    quad = p.clone()
    for k in ("W4", "b4"):
        learned.block(quad, k).zero_()
    lin = quad.clone()
    learned.fit_skip(lin, X, T, order=1)
    mse_quad, mse_lin = learned.evaluate(quad, Xv, Tv), learned.evaluate(lin, Xv, Tv)
    # the network's one-sector error is far below the skip connection's alone
    assert mse < mse_quad / 100 and mse_quad < mse_lin, (mse, mse_quad, mse_lin)

    rng = np.random.default_rng(4)
    n, turns = 512, 1000
    # Gaussian in the normalised phase space (sigma 0.3, inside radius 0.9),
    # energies across the range
    s = np.zeros((n, 5))
    s[:, :4] = 0.3 * rng.standard_normal((n, 4))
    for j in (0, 2):
        r = np.hypot(s[:, j], s[:, j + 1])
        s[:, j:j + 2] *= np.minimum(1.0, 0.9 / np.maximum(r, 1e-12))[:, None]
    s[:, 4] = rng.uniform(-0.9, 0.9, n)
    st = torch.from_numpy(s).cuda()
    P = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(s[:, 4])), device="cuda")
    phys = torch.cat([frame.to_phys(st, st[:, 4]), P[:, None]], 1)
    ref = learned.plain_track(frame, tracker, phys, turns, record=True)
    res = {}
    for name, prm in (("learned", p), ("second-order", quad), ("linear", lin)):
        lm = learned.LearnedSectorMap(frame, tracker, prm, audit_every=50, audit_frac=0.01, audit_tol=1e-5)
        res[name] = lm.track(phys, turns, record=True)
    q_ref = learned.tunes(ref["record"])
    e_ref = learned.betatron_emittance(frame, ref["record"][-1])
    out = {}
    for name, r in res.items():
        dq = np.abs(learned.tunes(r["record"]) - q_ref)
        de = np.abs(learned.betatron_emittance(frame, r["record"][-1]) / e_ref - 1).max()
        out[name] = (float(dq.max()), float(np.sqrt(np.mean(dq ** 2))), float(de), int(r["plain"].sum()))
    print("learned map (max dq, rms dq, emittance error, plain states):", out, "mse", mse, mse_quad, mse_lin)
    assert out["learned"][0] <= 1e-4, out
    assert out["learned"][2] <= 1e-2, out
    assert out["learned"][0] < out["second-order"][0] / 5, out


def test_graph_training_matches_eager():
    """The device-scheduled step replayed from one captured CUDA graph gives
    the parameters of the same steps run directly, bit for bit, and the
    device counter has advanced once per step."""
    from pyffa_b200 import learned
    B, steps = 512, 9
    rng = np.random.default_rng(21)
    X = np.zeros((B * steps, 8), np.float32)
    X[:, :5] = rng.uniform(-1, 1, (B * steps, 5))
    T = X.copy()
    T[:, :5] += 0.05 * rng.standard_normal((B * steps, 5)).astype(np.float32)
    dX, dT = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    p0 = torch.from_numpy(learned.init_params(3)).cuda()
    table = torch.linspace(1e-3, 2e-4, steps)
    out = []
    for graph in (False, True):
        p = p0.clone()
        tr = learned.Trainer(p, batch=B, lr_table=table)
        for i in range(steps):
            xb, tb = dX[i * B:(i + 1) * B], dT[i * B:(i + 1) * B]
            if graph:
                tr.graph_step(xb, tb)
            else:
                tr.step(xb.contiguous(), tb.contiguous(), 0.0)
        torch.cuda.synchronize()
        assert int(tr.counter.item()) == steps and tr.t == steps
        out.append((p.cpu().numpy(), tr.m.cpu().numpy(), tr.loss_part.cpu().numpy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    assert not np.array_equal(out[0][0], p0.cpu().numpy())          # the steps did move the parameters
