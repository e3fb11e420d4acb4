"""Launch-shape autotuner, host side (no GPU): the flag encoding shared with
include/ffa_cuda.h, the C-ABI's checks of the shape bits (made before any
CUDA call), the candidate lists, the residency model and the selection rule."""
import ctypes
import os
import re

import pytest

from pyffa_b200 import _lib, autotune, build

HEADER = os.path.join(build.REPO_DIR, "include", "ffa_cuda.h")


def test_shape_constants_match_header():
    text = open(HEADER).read()
    vals = {k: int(v, 0) for k, v in re.findall(r"\b(FFA_SHAPE_\w+)\s*=\s*(0x[0-9A-Fa-f]+|\d+)", text)}
    assert vals == {"FFA_SHAPE_TB_SHIFT": _lib.FFA_SHAPE_TB_SHIFT, "FFA_SHAPE_NREG_SHIFT": _lib.FFA_SHAPE_NREG_SHIFT,
                    "FFA_SHAPE_MASK": _lib.FFA_SHAPE_MASK}
    assert _lib.shape_flags(0, 0) == 0
    assert _lib.shape_flags(3, 3) == _lib.FFA_SHAPE_MASK
    assert _lib.shape_flags(2, 1) == (2 << 8) | (1 << 10)
    # shape bits are disjoint from the solver / precision / RF bits
    assert _lib.FFA_SHAPE_MASK & (_lib.FFA_RK4 | _lib.FFA_FP32C | _lib.FFA_RF_PHYSICAL_SUM) == 0
    with pytest.raises(ValueError):
        _lib.shape_flags(4, 0)


def _dummy_push_args(sc=False):
    """Descriptors that pass the argument checks; n = 0, so nothing is
    launched.  The field map is a zeroed host block larger than the library's
    map object, which the checks read (a map without field-error harmonics);
    no other pointer is dereferenced."""
    keep = ctypes.create_string_buffer(1 << 16)
    fake = ctypes.addressof(keep)
    rf = _lib.RFDesc()
    rf.ngaps = 1
    ap, cs = _lib.Aperture(), _lib.Consts()
    tab = _lib.StepTable()
    tab.drf = tab.acc = fake
    tab.nsteps = 10
    st = _lib.StateSoA()
    for name, _ in _lib.StateSoA._fields_:
        if sc or name not in ("sc_pre", "sc_pp", "e_pre_r", "e_pre_z", "e_pre_fi", "e_pp_r", "e_pp_z", "e_pp_fi"):
            setattr(st, name, fake)
    return keep, (fake, ctypes.byref(rf), ctypes.byref(ap), ctypes.byref(cs), ctypes.byref(tab), ctypes.byref(st))


def _push(flags, sc_step=0):
    keep, head = _dummy_push_args(sc=sc_step > 0)
    return _lib.lib().ffa_push(*head, 0, 0, 5, 1e-11, sc_step, flags, None, ctypes.addressof(keep))


def test_push_checks_shape_bits_before_any_cuda_call():
    B, R, F = _lib.FFA_BORIS, _lib.FFA_RK4, _lib.FFA_FP32C
    for t in range(4):
        assert _push(B | _lib.shape_flags(t, 0)) == 0          # every block size, float64 Boris
        for r in range(4):
            assert _push(F | _lib.shape_flags(t, r)) == 0      # every shape, FP32C Boris
    assert _push(B | _lib.shape_flags(0, 1)) == 4              # register caps: FP32C only
    assert _push(R | _lib.shape_flags(1, 0)) == 4              # RK4 takes the default shape only
    assert _push(R | F) == 0                                   # RK4 with the FP32C field
    assert _push(R | _lib.FFA_FP32) == 4                       # the float32 push is Boris-only
    assert _push(F | _lib.shape_flags(0, 2), sc_step=5) == 4   # and not with space charge
    assert _push(F | _lib.shape_flags(1, 0), sc_step=5) == 0   # block size with space charge: fine
    assert _push(B | (1 << 12)) == 1                           # unknown bit


def test_occupancy_query_checks_arguments_without_gpu():
    L = _lib.lib()
    b, t = ctypes.c_int32(), ctypes.c_int32()
    assert L.ffa_push_occupancy(0, 2, 1, None, ctypes.byref(t)) == 1
    assert L.ffa_push_occupancy(0, 9, 1, ctypes.byref(b), ctypes.byref(t)) == 1
    assert L.ffa_push_occupancy(_lib.FFA_RK4 | _lib.shape_flags(1, 0), 2, 0, ctypes.byref(b), ctypes.byref(t)) == 4
    assert L.ffa_push_occupancy(_lib.shape_flags(0, 3), 2, 0, ctypes.byref(b), ctypes.byref(t)) == 4


def test_candidates():
    c = autotune.candidates(fp32c=True)
    assert len(c) == 16 and len(set(c)) == 16 and (0, 0) in c
    assert autotune.candidates(fp32c=False) == [(0, 0), (1, 0), (2, 0), (3, 0)]
    assert autotune.candidates(fp32c=True, space_charge=True) == [(0, 0), (1, 0), (2, 0), (3, 0)]


def test_residency_model():
    m = autotune.modelled_warps_per_sm
    assert m(32, 80) == 24          # 6 warps of 2560 registers per 16384-register scheduler
    assert m(64, 72) == 28
    assert m(64, 64) == 32
    assert m(64, 56) == 36
    assert m(32, 56) == 32          # one-warp blocks: 32 blocks per SM at most
    assert m(256, 80) == 24
    assert m(256, 56) == 32         # 36 warps' registers, but whole 8-warp blocks: 4
    # every candidate against the runtime's occupancy calculator on a B200
    # (ffa_push_occupancy, FP32C Boris with crossing capture, map order 2)
    runtime = {(32, 80): 24, (64, 80): 24, (128, 80): 24, (256, 80): 24, (32, 72): 28, (64, 72): 28,
               (128, 72): 28, (256, 72): 24, (32, 64): 32, (64, 64): 32, (128, 64): 32, (256, 64): 32,
               (32, 56): 32, (64, 56): 36, (128, 56): 36, (256, 56): 32}
    assert {k: m(*k) for k in runtime} == runtime
    # the 256-energy scan bunch: 1.43 waves of the default shape, one of 36 warps
    assert abs(autotune.waves(162321, 24, 148) - 1.428) < 1e-3
    assert autotune.waves(162321, 36, 148) <= 1.0


def test_selection_rule():
    rows = [{"shape": (0, 0), "ms": 10.0}, {"shape": (1, 2), "ms": 9.9}, {"shape": (2, 3), "ms": 12.0}]
    assert autotune.select(rows, margin=0.02) == (0, 0)      # 1 % is within the margin
    rows[1]["ms"] = 9.0
    assert autotune.select(rows, margin=0.02) == (1, 2)
    rows[2]["ms"] = 8.0
    assert autotune.select(rows, margin=0.02) == (2, 3)
    assert autotune.select([{"shape": (0, 0), "ms": 1.0}], margin=0.0) == (0, 0)
    rows[2]["accepted"] = False                              # fastest, but its results differ
    assert autotune.select(rows, margin=0.02) == (1, 2)


def test_state_comparison():
    torch = pytest.importorskip("torch")
    a = torch.tensor([1.0, 2.0, float("nan"), -4.0], dtype=torch.float64)
    assert autotune.compare(a, a.clone()) == (True, 0.0)
    b = a.clone()
    b[1] = 2.0 * (1 + 1e-12)
    same, rel = autotune.compare(b, a)
    assert not same and abs(rel - 1e-12) < 1e-15
    c = a.clone()
    c[0] = float("nan")                                      # a NaN where there was none
    assert autotune.compare(c, a) == (False, float("inf"))


class _FakeEvent:
    """Stands in for torch.cuda.Event: the tuner reads e0.elapsed_time(e1)."""
    clock = [0.0]
    times = {}

    def __init__(self, enable_timing=False):
        self.t = None

    def record(self, stream=None):
        self.t = _FakeEvent.clock[0]

    def elapsed_time(self, other):
        return other.t - self.t


class _FakePusher:
    def __init__(self, times, differs):
        import torch
        self.flags = _lib.FFA_FP32C
        self.shape = (1, 1)                   # the caller's own shape, restored afterwards
        self.stream = type("S", (), {"synchronize": lambda s: None})()
        self.gp = type("G", (), {"Bmap": type("B", (), {"max_order": 2})()})()
        self.times, self.differs = times, differs
        self.calls = []
        self.state = torch.zeros(4, dtype=torch.float64)

    def push(self, clock, step0, nsteps, sc_step, xing=None):
        import torch
        self.calls.append(self.shape)
        _FakeEvent.clock[0] += self.times(self.shape, len(self.calls))
        self.state = torch.full((4,), 1.0 + (1e-12 if self.shape in self.differs else 0.0), dtype=torch.float64)


def _patch(monkeypatch):
    import contextlib
    import torch
    monkeypatch.setattr(torch.cuda, "Event", _FakeEvent)
    monkeypatch.setattr(torch.cuda, "stream", lambda s: contextlib.nullcontext())
    monkeypatch.setattr(autotune, "occupancy", lambda flags, order, xing: (12, 64))


def test_tune_push_bookkeeping(monkeypatch):
    _patch(monkeypatch)
    times = lambda shape, k: {(0, 0): 10.0, (2, 1): 8.0, (3, 3): 6.0}.get(shape, 9.9) + (5.0 if k % 3 == 1 else 0)
    pu = _FakePusher(times, differs={(3, 3)})
    resets = []
    res = autotune.tune_push(pu, None, 0, 100, reset=lambda: resets.append(1), snapshot=lambda: pu.state,
                             repeats=2)
    assert pu.shape == (1, 1)                                  # restored
    assert pu.calls[:3] == [(0, 0)] * 3 and len(pu.calls) == 3 * 16 and len(resets) == 3 * 16
    rows = {r["shape"]: r for r in res.rows}
    assert rows[(0, 0)]["ms"] == 10.0                          # the untimed first launch (+5) is not counted
    assert rows[(3, 3)]["identical"] is False and rows[(3, 3)]["max_rel_diff"] > 0
    assert rows[(3, 3)]["accepted"] is False and rows[(2, 1)]["accepted"] is True
    assert res.best == (2, 1) and abs(res.speedup - 10.0 / 8.0) < 1e-12
    # a tolerance admits the rounding-level shape, which is then the fastest
    pu2 = _FakePusher(times, differs={(3, 3)})
    res2 = autotune.tune_push(pu2, None, 0, 100, reset=lambda: None, snapshot=lambda: pu2.state, rtol=1e-9)
    assert res2.best == (3, 3)
    # cached by key: no launches the second time
    pu3 = _FakePusher(times, differs=set())
    r1 = autotune.tune_push(pu3, None, 0, 100, reset=lambda: None, snapshot=lambda: pu3.state, cache_key="k")
    n = len(pu3.calls)
    assert autotune.tune_push(pu3, None, 0, 100, cache_key="k") is r1 and len(pu3.calls) == n
    autotune._CACHE.clear()
