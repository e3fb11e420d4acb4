"""Launch-shape autotuner for the Boris pushers.

The push kernels give one particle to one thread for a whole launch, so a
launch is as long as its slowest wave of warps.  A launch shape is the pair
(threads per block, register cap per thread): the cap sets how many warps an
SM holds at once (its four schedulers have 16384 registers each, a warp
takes cap x 32 of them, and an SM holds at most 32 blocks and 64 warps), the
block size how those warps are grouped.  Together they decide how a bunch
of n particles falls into waves: the 162,321-particle bunch of a 256-energy
scan is 5,073 warps, 1.43 waves of the default shape (32 threads, 80
registers: 24 warps per SM), and one wave of 36 warps per SM (56 registers),
which spills more.  Which is faster depends on the spills and on how well
the extra warps hide latency, so the tuner measures instead of modelling:
every candidate pushes the same starting state for the same steps, timed
with CUDA events on the pusher's stream, and the fastest is kept unless it
beats the default by less than `margin`.

The block size does not touch the arithmetic.  The register cap changes
register allocation, and under a tight cap the code generator may also
place its multiply-add fusions differently (the source leaves it that
freedom), which moves results by rounding (measured: 7.5e-12 relative after 2500
steps at 56 registers; 72 and 64 were bit-identical).  So the tuner
compares each candidate's final state with the default shape's on the
tuning run (`snapshot`) and chooses only among the bit-identical ones, or,
for a caller that states a tolerance `rtol` (a fit, not a trajectory), among
those within it.

The candidates are the 4 block sizes x 4 register caps of the compensated
float32 pusher without space charge, and the 4 block sizes of the others
(their kernels are built with the default cap only).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

from . import _lib

SM_REGISTERS_PER_SCHEDULER = 16384
SM_MAX_BLOCKS = 32
SM_MAX_WARPS = 64


def candidates(fp32c: bool, space_charge: bool = False) -> list[tuple[int, int]]:
    """(threads index, register-cap index) pairs the library builds."""
    caps = range(len(_lib.SHAPE_NREGS)) if fp32c and not space_charge else [0]
    return [(t, r) for r in caps for t in range(len(_lib.SHAPE_THREADS))]


def modelled_warps_per_sm(threads: int, nreg: int) -> int:
    """Resident warps per SM from the register split over the four
    schedulers and the block and warp limits (the runtime's figure, from
    ffa_push_occupancy, is reported beside it)."""
    per_sched = SM_REGISTERS_PER_SCHEDULER // (32 * nreg)
    wpb = threads // 32
    blocks = min(SM_MAX_BLOCKS, (4 * per_sched) // wpb)
    return min(SM_MAX_WARPS, blocks * wpb)


def waves(n: int, warps_per_sm: int, sms: int) -> float:
    """Warps of an n-particle bunch over the warps the GPU holds at once."""
    return (n + 31) // 32 / max(1, warps_per_sm * sms)


def occupancy(flags: int, max_order: int, crossing: bool) -> tuple[int, int]:
    """(resident blocks per SM, threads per block) from the runtime."""
    blocks, tb = ctypes.c_int32(), ctypes.c_int32()
    _lib.check(_lib.lib().ffa_push_occupancy(flags, max_order, int(crossing), ctypes.byref(blocks),
                                             ctypes.byref(tb)), "ffa_push_occupancy")
    return blocks.value, tb.value


@dataclass
class TuneResult:
    best: tuple[int, int]
    default_ms: float
    best_ms: float
    rows: list = field(default_factory=list)

    @property
    def speedup(self) -> float:
        return self.default_ms / self.best_ms

    def report(self) -> dict:
        t, r = self.best
        return {"chosen": {"threads": _lib.SHAPE_THREADS[t], "max_regs": _lib.SHAPE_NREGS[r]},
                "speedup_vs_default": self.speedup, "candidates": self.rows}


def select(rows: list[dict], margin: float) -> tuple[int, int]:
    """The fastest accepted candidate (rows without an "accepted" entry are
    accepted), or the default (0, 0) when the fastest beats it by less than
    the fraction `margin` (timing noise is not a reason to leave the
    default)."""
    default = next(r for r in rows if r["shape"] == (0, 0))
    best = min((r for r in rows if r.get("accepted", True)), key=lambda r: r["ms"])
    return best["shape"] if best["ms"] < (1.0 - margin) * default["ms"] else (0, 0)


def compare(a, b) -> tuple[bool, float]:
    """(bit-identical, largest relative difference) of two state tensors;
    NaN must sit in the same places in both (else the difference is inf)."""
    import torch
    if a.shape != b.shape:
        return False, float("inf")
    na, nb = torch.isnan(a), torch.isnan(b)
    if not bool((na == nb).all()):
        return False, float("inf")
    ok = ~na
    same = bool((a[ok] == b[ok]).all())
    if same:
        return True, 0.0
    rel = (a[ok] - b[ok]).abs() / b[ok].abs().clamp_min(1e-300)
    return False, float(rel.max())


_CACHE: dict = {}


def tune_push(pusher, clock, step0: int, nsteps: int, xing=None, reset=None, count=None, repeats: int = 2,
              margin: float = 0.02, cands=None, cache_key=None, snapshot=None, rtol: float = 0.0) -> TuneResult:
    """Times `repeats` launches of `nsteps` steps from absolute step `step0`
    for every candidate launch shape of `pusher` (after one untimed launch
    each, which also loads the kernel) and returns the choice; the pusher's
    own shape is left as it was.  reset(): enqueued before every launch to
    put the bunch back in its starting state (the pushes advance it);
    count: the crossing-record counter to clear before a launch that
    captures crossings; snapshot(): a tensor of the pushed state, compared
    with the default shape's (needs `reset`; default: the bunch's coordinate
    columns); a candidate is accepted if bit-identical, or with rtol > 0 if
    within rtol relative everywhere.  A cache_key reuses an earlier result."""
    import torch
    if cache_key is not None and cache_key in _CACHE:
        return _CACHE[cache_key]
    if cands is None:
        fp32c = bool(pusher.flags & _lib.FFA_FP32C) and not (pusher.flags & _lib.FFA_RK4)
        cands = candidates(fp32c) if not (pusher.flags & _lib.FFA_RK4) else [(0, 0)]
    cands = [(0, 0), *[c for c in cands if c != (0, 0)]]
    if snapshot is None and reset is not None and hasattr(pusher.bunch, "cols"):
        def snapshot():
            import torch
            return torch.stack([pusher.bunch.cols[k] for k in ("r", "vr", "z", "vz", "fi", "f5", "rf")])
    ref = None
    st = pusher.stream
    saved = pusher.shape
    rows = []
    max_order = int(getattr(pusher.gp.Bmap, "max_order", 0))
    try:
        for c in cands:
            pusher.shape = c
            times = []
            for k in range(repeats + 1):
                with torch.cuda.stream(st):
                    if reset is not None:
                        reset()
                    if count is not None:
                        count.zero_()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    pusher.push(clock, step0, nsteps, 0, xing=xing)
                    e1.record(st)
                st.synchronize()
                if k:
                    times.append(e0.elapsed_time(e1))
            threads, nreg = _lib.SHAPE_THREADS[c[0]], _lib.SHAPE_NREGS[c[1]]
            row = {"shape": c, "threads": threads, "max_regs": nreg, "ms": min(times),
                   "warps_per_sm_model": modelled_warps_per_sm(threads, nreg)}
            if snapshot is not None and reset is not None:
                with torch.cuda.stream(st):
                    snap = snapshot().clone()
                st.synchronize()
                if ref is None:
                    ref = snap
                same, rel = compare(snap, ref)
                row.update(identical=same, max_rel_diff=rel, accepted=same or rel <= rtol)
            blocks, tb = occupancy(pusher.flags | _lib.shape_flags(*c), max_order, xing is not None)
            row["warps_per_sm"] = blocks * tb // 32
            rows.append(row)
    finally:
        pusher.shape = saved
    best = select(rows, margin)
    res = TuneResult(best=best, default_ms=next(r["ms"] for r in rows if r["shape"] == (0, 0)),
                     best_ms=next(r["ms"] for r in rows if r["shape"] == best), rows=rows)
    if cache_key is not None:
        _CACHE[cache_key] = res
    return res
