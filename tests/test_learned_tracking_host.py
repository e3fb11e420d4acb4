"""Learned-map tracking orchestration on the CPU: domain fallback, audits
and the hand-over to the plain tracker, with the network and the tracker
replaced by exact rotations in the normalised frame (no GPU, no library
call)."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from pyffa_b200 import learned  # noqa: E402

MU = (2 * math.pi * 3.6 / 12, 2 * math.pi * 0.78 / 12)


def _frame():
    return learned.SectorFrame((300.0, 600.0), [8.5, 0.2], [0.01, 0.0], (0.3, 2.0), (-0.2, 3.0), (10e-3, 5e-3), 12)


def _rotate(s, mu, k):
    out = s.clone()
    for j, m in ((0, mu[0]), (2, mu[1])):
        c, sn = math.cos(k * m), math.sin(k * m)
        out[:, j] = c * s[:, j] + sn * s[:, j + 1]
        out[:, j + 1] = -sn * s[:, j] + c * s[:, j + 1]
    return out


class RotTracker:
    """Plain-tracker stand-in: the exact rotation in the frame."""

    def __init__(self, frame):
        self.frame, self.dev, self.nsectors, self.calls = frame, torch.device("cpu"), 12, []

    def run(self, x0, n_sectors=1):
        self.calls.append((x0.shape[0], n_sectors))
        s = self.frame.to_norm(x0)
        return self.frame.to_phys(_rotate(s, MU, n_sectors), s[:, 4])


class RotMap(learned.LearnedSectorMap):
    """Network stand-in: a rotation (optionally off by `dmu`), with the
    kernel's domain rule."""
    dmu = 0.0

    def pack(self):
        pass

    def error_flag(self):
        return 0

    def apply(self, state, n_apply, applied=None, radius2=None):
        r2 = self.radius2 if radius2 is None else radius2
        cnt = torch.zeros(state.shape[0], dtype=torch.int32)
        act = torch.ones(state.shape[0], dtype=torch.bool)
        for _ in range(n_apply):
            inside = ((state[:, 0] ** 2 + state[:, 1] ** 2 <= r2) & (state[:, 2] ** 2 + state[:, 3] ** 2 <= r2)
                      & (state[:, 4].abs() <= 1))
            act &= inside
            nxt = _rotate(state.double(), (MU[0] + self.dmu, MU[1]), 1).float()
            state[act, :4] = nxt[act, :4]
            cnt += act.int()
        if applied is not None:
            applied.copy_(cnt)


def _bunch(frame, n, seed, radius=0.9):
    s = torch.from_numpy(learned.sample_domain(n, np.random.default_rng(seed), radius))
    P = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(s[:, 4].numpy())))
    return torch.cat([frame.to_phys(s, s[:, 4]), P[:, None]], 1), s


def test_learned_path_without_fallback():
    frame = _frame()
    tr = RotTracker(frame)
    lm = RotMap(frame, tr, torch.zeros(learned.N_PARAMS), audit_every=50, audit_frac=0.05, audit_tol=1e-5)
    phys, s = _bunch(frame, 200, 1)
    res = lm.track(phys, 120)
    assert not res["plain"].any()
    exp = frame.to_phys(_rotate(s, MU, 120 * 12), s[:, 4])
    assert (res["phys"] - exp).abs().max().item() < 1e-6
    # audits at turns 50 and 100, 5% of the states each, all passing
    assert [(a[0], a[1], a[2]) for a in res["audits"]] == [(50, 10, 0), (100, 10, 0)]
    # the plain tracker ran only the audit sectors
    assert tr.calls == [(10, 1), (10, 1)]


def test_out_of_domain_states_go_to_the_plain_tracker():
    frame = _frame()
    tr = RotTracker(frame)
    lm = RotMap(frame, tr, torch.zeros(learned.N_PARAMS), audit_every=50, audit_frac=0.0)
    phys, s = _bunch(frame, 50, 2)
    phys2, s2 = phys.clone(), s.clone()
    # state 0: amplitude 1.2 (outside), state 1: energy beyond the range
    s2[0, 0], s2[0, 1] = 1.2, 0.0
    s2[1, 4] = 1.2
    P = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(s2[:, 4].numpy())))
    phys2 = torch.cat([frame.to_phys(s2, s2[:, 4]), P[:, None]], 1)
    res = lm.track(phys2, 30, record=True)
    assert res["plain"].tolist()[:2] == [True, True] and not res["plain"][2:].any()
    exp = frame.to_phys(_rotate(s2, MU, 30 * 12), s2[:, 4])
    assert (res["phys"] - exp).abs().max().item() < 1e-6
    assert res["record"].shape == (31, 50, 4)
    # the record of a plain state is its normalised state every turn
    assert np.allclose(res["record"][7, 0], _rotate(s2[:1], MU, 84)[0, :4].numpy(), atol=1e-6)


def test_failed_audit_hands_states_over():
    frame = _frame()
    tr = RotTracker(frame)
    lm = RotMap(frame, tr, torch.zeros(learned.N_PARAMS), audit_every=10, audit_frac=0.5, audit_tol=1e-9, seed=3)
    lm.dmu = 1e-4                       # the "network" is off: every audit fails
    phys, s = _bunch(frame, 40, 4)
    res = lm.track(phys, 20)
    a1, a2 = res["audits"]
    assert a1[:3] == (10, 20, 20) and a2[:3] == (20, 10, 10)
    assert int(res["plain"].sum()) == 30


def test_save_and_load_round_trip(tmp_path):
    frame = _frame()
    p = learned.init_params(5)
    path = str(tmp_path / "map.npz")
    learned.save(path, torch.from_numpy(p), frame)
    p2, f2 = learned.load(path)
    assert np.array_equal(p2, p)
    s = torch.from_numpy(learned.sample_domain(50, np.random.default_rng(6)))
    a = frame.to_phys(s, s[:, 4])
    b = f2.to_phys(s, s[:, 4])
    assert torch.equal(a, b) and f2.R == frame.R and f2.nsectors == 12
