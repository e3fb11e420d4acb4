"""Batched closed-orbit and tune scan with the compensated float32 pusher.

Many independent instances (one energy each, a few to thousands of
particles with small offsets around a guessed orbit) run as ONE bunch
through the FP32C Boris pusher: every launch advances all instances, so the
load of small and large instances is balanced particle by particle.  Per
iteration the bunch is pushed for `turns` turns of the slowest instance, the
azimuth-0 crossings of every particle (ffa_push_crossing; the state at the
azimuth from a cubic Hermite interpolation of the step in Cartesian
coordinates) are paired turn to turn inside the push kernel, which adds each
pair to its instance's normal equations of the least-squares one-turn map
x' = M x + b (per transverse plane, over all of the instance's particles and
turns, float64); the map is solved on the host.  Its fixed point
(I - M)^-1 b is the Newton update of the closed orbit; the phase advance of
M (trace, with the sign of M12 fixing the half plane) is the fractional tune.
The next iteration restarts the instances around the updated orbits.

The reference's counterpart is the per-energy closed-orbit search in the
azimuth domain (FFAG_SearchSEO, src/FFAG_track.py:1142-1586: fixed-point
averaging and a finite-difference Newton step on the one-sector map, tunes
from the transfer-matrix trace, GetQrQz src/FFAG_track.py:1257-1309); this
scan does the same with time-domain tracking of particle ensembles, which is
what a tracking code sees, for all energies in one launch sequence.
"""
from __future__ import annotations

import math

import numpy as np

from .constants import FFAG_ConversionTools


def crossing_states(rec, dt, iterations=3, target=0.0):
    """States (k, 4) = r, vr, z, vz at the azimuth `target` (rad) of crossing
    records (k, 23).

    The pre- and post-step states are taken to Cartesian coordinates (x axis
    along the target azimuth) and the
    step is interpolated as a cubic Hermite curve in time (positions and
    velocities at both ends), the crossing time found by Newton on y(tau) = 0
    from the linear estimate; velocities are interpolated linearly.  Near
    azimuth 0 the orbit runs through a drift, where this is exact, whereas a
    linear interpolation of r in the azimuth misses by r'' dphi^2 / 8 (about
    80 um at 720 steps per turn)."""
    import torch

    def cart(o):
        r, vr, z, vz, fi, f5 = (rec[:, o + j] for j in range(6))
        c, s_ = torch.cos(fi - target), torch.sin(fi - target)
        vf = r * f5
        return r * c, r * s_, z, vr * c - vf * s_, vr * s_ + vf * c, vz

    X0, Y0, Z0, VX0, VY0, VZ0 = cart(4)
    X1, Y1, Z1, VX1, VY1, VZ1 = cart(11)
    tau = Y0 / (Y0 - Y1)
    for _ in range(iterations):
        t2, t3 = tau * tau, tau * tau * tau
        y = (2 * t3 - 3 * t2 + 1) * Y0 + (t3 - 2 * t2 + tau) * VY0 * dt + (3 * t2 - 2 * t3) * Y1 + (t3 - t2) * VY1 * dt
        dy = (6 * t2 - 6 * tau) * Y0 + (3 * t2 - 4 * tau + 1) * VY0 * dt + (6 * tau - 6 * t2) * Y1 + (3 * t2 - 2 * tau) * VY1 * dt
        tau = tau - y / dy
    t2, t3 = tau * tau, tau * tau * tau
    h00, h10, h01, h11 = 2 * t3 - 3 * t2 + 1, t3 - 2 * t2 + tau, 3 * t2 - 2 * t3, t3 - t2
    X = h00 * X0 + h10 * VX0 * dt + h01 * X1 + h11 * VX1 * dt
    Z = h00 * Z0 + h10 * VZ0 * dt + h01 * Z1 + h11 * VZ1 * dt
    VX = VX0 + tau * (VX1 - VX0)
    VZ = VZ0 + tau * (VZ1 - VZ0)
    return torch.stack([X, VX, Z, VZ], 1)


def _lib_record_bytes():
    from . import _lib
    return 8 * _lib.CROSSING_RECORD


def accumulate_crossings(p, step, x, gv, inst, nsteps, last, has, S, Y, crossings, scale=None):
    """Adds one launch's crossings to the per-instance sums.

    p (k,) particle indices, step (k,) absolute steps, x (k, 4) states at the
    azimuth (r, vr, z, vz), in any order.  The states are taken relative to
    the guessed orbit gv[instance] and multiplied by scale[instance] (4
    factors that make the coordinates of order one and the normal equations
    well conditioned; None: 1), and each is paired with the same particle's
    previous crossing (this launch, or `last` from earlier ones).
    S[plane, i] += f f^T and Y[plane, i] += x' f^T with f = (x, x_dot, 1) of
    the earlier crossing and x' the later one; crossings[i] counts records."""
    import torch
    k = p.shape[0]
    x = x - gv[inst[p]]
    if scale is not None:
        x = x * scale[inst[p]]
    order = torch.argsort(p * (nsteps + 2) + step)
    p, x = p[order], x[order]
    same = torch.zeros(k, dtype=torch.bool, device=x.device)
    same[1:] = p[1:] == p[:-1]
    prev = torch.empty_like(x)
    prev[1:] = x[:-1]
    first = ~same
    prev[first] = last[p[first]]
    ok = same | (first & has[p])
    xp, xn, ip = prev[ok], x[ok], inst[p[ok]]
    for pl in (0, 1):
        f = torch.cat([xp[:, 2 * pl:2 * pl + 2], torch.ones_like(xp[:, :1])], 1)
        S[pl].index_add_(0, ip, f[:, :, None] * f[:, None, :])
        Y[pl].index_add_(0, ip, xn[:, 2 * pl:2 * pl + 2, None] * f[:, None, :])
    crossings.index_add_(0, inst[p], torch.ones(k, dtype=crossings.dtype, device=x.device))
    lastocc = torch.ones(k, dtype=torch.bool, device=x.device)
    lastocc[:-1] = p[1:] != p[:-1]
    last[p[lastocc]] = x[lastocc]
    has[p[lastocc]] = True


def accumulate_crossings_fixed(rec, count, dt, gv, inst_ext, nsteps, last, has, S, Y, crossings, scale):
    """accumulate_crossings over a whole record buffer (C, 23) of which the
    first `count` (device scalar) rows are valid, with no host read-back and
    no data-dependent shapes (capturable in a CUDA graph).  Invalid rows go to
    a dummy particle N (inst_ext[N] = I, the dummy instance: gv[I] = 0,
    scale[I] = 1, rows I of S, Y, crossings and N of last, has unused)."""
    import torch
    C = rec.shape[0]
    N = inst_ext.shape[0] - 1
    I = gv.shape[0] - 1
    valid = torch.arange(C, device=rec.device) < count
    p = torch.where(valid, rec[:, 1].long(), N)
    step = torch.where(valid, rec[:, 2].long(), 0)
    x = torch.where(valid[:, None], crossing_states(rec, dt), torch.zeros((), dtype=rec.dtype, device=rec.device))
    ii = inst_ext[p]
    x = (x - gv[ii]) * scale[ii]
    order = torch.argsort(p * (nsteps + 2) + step)
    p, x = p[order], x[order]
    ii = inst_ext[p]
    same = torch.zeros(C, dtype=torch.bool, device=rec.device)
    same[1:] = p[1:] == p[:-1]
    prev = torch.empty_like(x)
    prev[1:] = x[:-1]
    first = ~same
    prev = torch.where(first[:, None], last[p], prev)
    ok = same | (first & has[p])
    ip = torch.where(ok, ii, I)
    for pl in (0, 1):
        f = torch.cat([prev[:, 2 * pl:2 * pl + 2], torch.ones_like(prev[:, :1])], 1)
        S[pl].index_add_(0, ip, f[:, :, None] * f[:, None, :])
        Y[pl].index_add_(0, ip, x[:, 2 * pl:2 * pl + 2, None] * f[:, None, :])
    crossings.index_add_(0, ii, torch.ones(C, dtype=crossings.dtype, device=rec.device))
    lastocc = torch.ones(C, dtype=torch.bool, device=rec.device)
    lastocc[:-1] = p[1:] != p[:-1]
    idx = torch.where(lastocc, p, N)
    last.index_copy_(0, idx, x)
    has.index_fill_(0, idx, True)


def unpack_fit_sums(sums):
    """S (2, I, 3, 3) and Y (2, I, 2, 3) of accumulate_crossings, and the
    crossing counts (I,), from the (I, 25) sums a push accumulates at
    crossing time (ffa_crossing.fit_sums): per plane the upper triangle of
    f f^T (f0 f0, f0 f1, f0, f1 f1, f1, 1) then x' f^T row by row; the
    crossings last."""
    sums = np.asarray(sums, np.float64)
    I = sums.shape[0]
    S = np.empty((2, I, 3, 3))
    Y = np.empty((2, I, 2, 3))
    for pl in (0, 1):
        q = sums[:, 12 * pl:12 * pl + 12]
        S[pl, :, 0, 0], S[pl, :, 0, 1], S[pl, :, 0, 2] = q[:, 0], q[:, 1], q[:, 2]
        S[pl, :, 1, 1], S[pl, :, 1, 2], S[pl, :, 2, 2] = q[:, 3], q[:, 4], q[:, 5]
        S[pl, :, 1, 0], S[pl, :, 2, 0], S[pl, :, 2, 1] = q[:, 1], q[:, 2], q[:, 4]
        Y[pl] = q[:, 6:12].reshape(I, 2, 3)
    return S, Y, sums[:, 24].copy()


def fit_one_turn(S, Y, cond_max=1e14):
    """float64 least-squares one-turn map per instance and plane from the sums
    of accumulate_crossings: returns the fixed point offsets (I, 4), the
    fractional tunes (I, 2) and a validity mask (I,)."""
    I = S.shape[1]
    tunes = np.full((I, 2), np.nan)
    fix = np.zeros((I, 4))
    good = np.ones(I, dtype=bool)
    for i in range(I):
        for pl in (0, 1):
            A, B = S[pl, i], Y[pl, i]
            if not np.all(np.isfinite(A)) or np.linalg.cond(A) > cond_max:
                good[i] = False
                continue
            W = np.linalg.solve(A.T, B.T).T                       # B A^-1
            M, bb = W[:, :2], W[:, 2]
            fix[i, 2 * pl:2 * pl + 2] = np.linalg.solve(np.eye(2) - M, bb)
            c = np.clip(0.5 * np.trace(M), -1.0, 1.0)
            mu = math.acos(c) if M[0, 1] > 0 else 2 * math.pi - math.acos(c)
            tunes[i, pl] = mu / (2 * math.pi)
    return fix, tunes, good


def instance_counts(n_instances=256, max_count=4096, seed=0):
    """ceil(exp(U(0, ln max_count))) particles per instance (seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.ceil(np.exp(rng.uniform(0.0, math.log(max_count), n_instances))).astype(np.int64)


class BatchedOrbitScan:
    """All instances of a scan in one device bunch.

    gp: FFAG_GlobalParameters with the field map and an Emap (RF off);
    energies (I,) MeV; counts (I,) particles per instance; guesses r0 (I,)
    [m] and pr0 (I,) (p-format angle) of the closed orbit at azimuth 0 and
    its length `perimeter` (I,) [m]; sigma: Gaussian offset in r and z [m].
    The time step is the fastest instance's revolution time / steps_per_turn;
    an iteration lasts `turns` turns of the slowest instance.  autotune: the
    push's launch shape (threads per block, register cap) is picked by
    timing the candidates on the scan's own bunch before the first iteration
    (autotune.tune_push; `tuning` holds the table), else the default; shapes
    whose states differ from the default's by more than tune_rtol (relative)
    on the tuning run are not chosen.  The scan fits maps to many crossings,
    so rounding-level differences (1e-11) are accepted by default.
    accumulate="kernel": the push kernel itself adds each crossing to its
    instance's normal equations (ffa_crossing.fit_sums), so the whole
    iteration is one push launch whose memory is 25 doubles per instance and
    4 doubles + 1 byte per particle, whatever the number of turns.
    accumulate="records": the crossing records are written to a device
    buffer and reduced into the same sums by accumulate_crossings_fixed
    (kept to check the kernel's sums); persistent: the whole iteration is one
    push launch, its records held in one buffer (about 1.8 KB per particle
    and turn-bound of crossings: 10 GB for 162k particles over 200 turns),
    when that buffer and the accumulation's temporaries (taken as 3x the
    buffer) fit in half the free device memory; otherwise, and with
    persistent=False, launches of the longest length whose records fit that
    memory (at most 5 records per particle without `persistent`)."""

    def __init__(self, gp, energies, counts, r0, pr0, perimeter, sigma=0.5e-3, steps_per_turn=720, turns=200,
                 seed=0, device=None, autotune=True, tune_steps=1000, tune_rtol=1e-9, persistent=True,
                 accumulate="kernel"):
        import torch
        if accumulate not in ("kernel", "records"):
            raise ValueError(f"accumulate must be 'kernel' or 'records', not {accumulate!r}")
        self.accumulate = accumulate
        self.gp = gp
        self.persistent = bool(persistent)
        self.autotune = bool(autotune)
        self.tune_steps = int(tune_steps)
        self.tune_rtol = float(tune_rtol)
        self.tuning = None
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.E = np.asarray(energies, np.float64)
        self.counts = np.asarray(counts, np.int64)
        self.I = len(self.E)
        self.r = np.asarray(r0, np.float64).copy()
        self.pr = np.asarray(pr0, np.float64).copy()
        self.z = np.zeros(self.I)
        self.pz = np.zeros(self.I)
        self.conv = FFAG_ConversionTools()
        v = self.conv.Ek2v(self.E)
        self.T = np.asarray(perimeter, np.float64) / v
        self.dt = float(self.T.min() / steps_per_turn)
        self.turns = int(turns)
        self.steps = int(math.ceil(self.turns * self.T.max() / self.dt))
        self.inst = np.repeat(np.arange(self.I), self.counts)
        self.N = int(self.counts.sum())
        rng = np.random.Generator(np.random.PCG64(seed))
        self.g = sigma * rng.standard_normal((self.N, 2))    # r and z offsets, fixed over the iterations
        self.history = []
        self._dev_state = None
        self._graph = None

    # ------------------------------------------------------------ bunch
    def _vformat(self):
        a = np.zeros((self.N, 16))
        i = self.inst
        a[:, 0] = self.r[i] + self.g[:, 0]
        a[:, 1] = self.pr[i]
        a[:, 2] = self.z[i] + self.g[:, 1]
        a[:, 3] = self.pz[i]
        a[:, 5] = self.E[i]
        a[:, 15] = np.arange(self.N)
        v = self.conv.ConvertPrzek2Vrzek_boris(a)
        v[:, 7] = 1.0
        v[:, 8] = 1.0
        return v

    def _guess_v(self):
        """v-format (r, vr, z, vz) of the guessed orbits."""
        a = np.zeros((self.I, 16))
        a[:, 0], a[:, 1], a[:, 2], a[:, 3], a[:, 5] = self.r, self.pr, self.z, self.pz, self.E
        v = self.conv.ConvertPrzek2Vrzek_boris(a)
        return v[:, [0, 1, 2, 3]]

    # ------------------------------------------------------------ one iteration
    def _setup(self):
        """Device buffers of an iteration, allocated once: the bunch, the
        pusher on a private stream, the crossing buffer for the longest
        launch, the per-instance sums (with a dummy instance I and a dummy
        particle N for the fixed-shape accumulation)."""
        import torch
        from .track import CrossingCapture, Pusher, StepClock, _EphemeralBunch
        dev = self.dev
        f64 = dict(dtype=torch.float64, device=dev)
        st = type("ScanState", (), {})()
        st.stream = torch.cuda.Stream(dev)
        st.bunch = _EphemeralBunch(self._vformat(), "Boris", dev)
        st.pusher = Pusher(st.bunch, self.gp, "Boris", "fp32c")
        st.pusher.order_every = 0     # one thread order for the scan's life (graph replays read it)
        st.pusher.stream = st.stream
        st.clock = StepClock(0.0, self.dt, self.gp.Emap, "Boris", dev)
        st.clock.ensure(self.steps + 1)
        unit = np.ones((self.I + 1, 4))
        unit[:self.I, 0] = unit[:self.I, 2] = 1e-3
        unit[:self.I, 1] = unit[:self.I, 3] = 1e-3 * self.conv.Ek2v(self.E)
        st.unit = unit[:self.I]
        st.scale = torch.as_tensor(1.0 / unit, **f64)
        st.gv = torch.zeros((self.I + 1, 4), **f64)
        st.inst = torch.as_tensor(np.concatenate([self.inst, [self.I]]), device=dev)
        st.last = torch.zeros((self.N + 1, 4), **f64)
        st.has = torch.zeros(self.N + 1, dtype=torch.bool, device=dev)
        st.S = torch.zeros((2, self.I + 1, 3, 3), **f64)
        st.Y = torch.zeros((2, self.I + 1, 2, 3), **f64)
        st.crossings = torch.zeros(self.I + 1, **f64)
        st.maxk = torch.zeros(1, dtype=torch.int64, device=dev)
        if self.accumulate == "kernel":
            from . import _lib
            st.cap = None
            st.L = self.steps
            st.fit_inst = torch.as_tensor(self.inst.astype(np.int32), device=dev)
            st.fit_last = torch.zeros((self.N, 4), **f64)
            st.fit_has = torch.zeros(self.N, dtype=torch.uint8, device=dev)
            st.sums = torch.zeros((self.I, _lib.FIT_SUMS), **f64)
            x = _lib.Crossing()
            x.ntargets = 1
            x.target[0] = 0.0
            x.fit_instance = st.fit_inst.data_ptr()
            x.fit_centre = st.gv.data_ptr()
            x.fit_scale = st.scale.data_ptr()
            x.fit_last = st.fit_last.data_ptr()
            x.fit_has = st.fit_has.data_ptr()
            x.fit_sums = st.sums.data_ptr()
            st.xing = x
        else:
            st.cap = CrossingCapture(st.bunch, [0.0], self.gp, self.dt)
            st.L = self._launch_steps(st.cap)
            st.xing = st.cap.prepare(st.L)
            st.rows = st.cap.buf.view(-1, 23)[:st.cap.x.capacity]
        st.launches = len(range(0, self.steps, st.L))
        self._dev_state = st
        if self.autotune:
            self._tune()

    def _tune(self):
        """Times every launch shape on the first `tune_steps` steps of the
        scan's starting bunch, with crossing capture as in an iteration, and
        sets the fastest on the pusher."""
        import ctypes
        from . import _lib, autotune
        st = self._dev_state
        b = st.bunch

        def reset():
            _lib.check(_lib.lib().ffa_aos_to_soa(b.aos.data_ptr(), b.n, ctypes.byref(b.soa()),
                                                 st.stream.cuda_stream), "ffa_aos_to_soa")
            if st.cap is None:
                for t in (st.sums, st.fit_last, st.fit_has):
                    t.zero_()
        res = autotune.tune_push(st.pusher, st.clock, 0, min(st.L, self.tune_steps, self.steps), xing=st.xing,
                                 reset=reset, count=None if st.cap is None else st.cap.count,
                                 rtol=self.tune_rtol)
        st.pusher.shape = res.best
        self.tuning = res

    def _launch_steps(self, cap):
        """Steps per push launch: the whole iteration when its records fit
        (see the class notes), else the longest launch that fits."""
        import torch
        short = cap.max_steps()
        if not self.persistent:
            return min(short, self.steps)
        free, _ = torch.cuda.mem_get_info(self.dev)
        budget = free // 2

        def need(L):    # record buffer + 3x for the accumulation's temporaries
            per = 2 + int(np.ceil(L * cap.dt * cap.f_max / (2 * np.pi)))
            return 4 * cap.bunch.n * cap.x.ntargets * per * _lib_record_bytes()
        if need(self.steps) <= budget:
            return self.steps
        lo, hi = min(short, self.steps), self.steps
        while hi - lo > 1:                  # longest launch within the budget
            mid = (lo + hi) // 2
            lo, hi = (mid, hi) if need(mid) <= budget else (lo, mid)
        return lo

    def _body(self):
        """The work of one iteration, enqueued on the scan's stream: AoS ->
        SoA, then the push with the kernel's own accumulation, or for every
        launch the push with crossing capture and the accumulation of its
        records."""
        import ctypes
        from . import _lib
        st = self._dev_state
        b = st.bunch
        _lib.check(_lib.lib().ffa_aos_to_soa(b.aos.data_ptr(), b.n, ctypes.byref(b.soa()), st.stream.cuda_stream),
                   "ffa_aos_to_soa")
        if st.cap is None:
            for t in (st.sums, st.fit_last, st.fit_has):
                t.zero_()
            st.pusher.push(st.clock, 0, self.steps, 0, xing=st.xing)
            return
        for t in (st.S, st.Y, st.crossings, st.last, st.has, st.maxk):
            t.zero_()
        for s0 in range(0, self.steps, st.L):
            ns = min(st.L, self.steps - s0)
            st.cap.count.zero_()
            st.pusher.push(st.clock, s0, ns, 0, xing=st.xing)
            st.maxk.copy_(st.maxk.maximum(st.cap.count))
            accumulate_crossings_fixed(st.rows, st.cap.count, self.dt, st.gv, st.inst, self.steps, st.last, st.has,
                                       st.S, st.Y, st.crossings, st.scale)

    def _body_direct(self):
        """The iteration without a graph: each launch's record count is read
        back and only those records are accumulated."""
        import ctypes
        from . import _lib
        st = self._dev_state
        if st.cap is None:
            self._body()
            return
        b = st.bunch
        _lib.check(_lib.lib().ffa_aos_to_soa(b.aos.data_ptr(), b.n, ctypes.byref(b.soa()), st.stream.cuda_stream),
                   "ffa_aos_to_soa")
        for t in (st.S, st.Y, st.crossings, st.last, st.has, st.maxk):
            t.zero_()
        for s0 in range(0, self.steps, st.L):
            ns = min(st.L, self.steps - s0)
            st.cap.count.zero_()
            st.pusher.push(st.clock, s0, ns, 0, xing=st.xing)
            k = int(st.cap.count.item())
            st.maxk.fill_(max(int(st.maxk.item()), k))
            if k == 0 or k > st.cap.x.capacity:
                continue
            rec = st.rows[:k]
            accumulate_crossings(rec[:, 1].long(), rec[:, 2].long(), crossing_states(rec, self.dt), st.gv, st.inst,
                                 self.steps, st.last, st.has, st.S, st.Y, st.crossings, st.scale)

    def iterate(self, graph=True):
        """One push of all instances and the float64 update; returns the
        iteration record (orbit change, tunes, particle-turns, device time).
        With accumulate="kernel" an iteration is one push launch either way.
        With "records", graph=False: the launches run directly, each launch's
        records counted on the host and accumulated ("direct"); graph=True:
        the fixed-shape accumulation over the whole record buffer, which has
        no host read-back.  With graph=True the first iteration runs directly
        (it is also the warm-up, "captured") and is captured as one CUDA
        graph, which later iterations replay after uploading their starting
        states and guesses ("graph")."""
        import torch
        if self._dev_state is None:
            self._setup()
        st = self._dev_state
        with torch.cuda.stream(st.stream):
            st.bunch.aos.copy_(torch.from_numpy(self._vformat()))
            st.gv[:self.I].copy_(torch.from_numpy(self._guess_v()))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st.stream)
            if not graph:
                self._body_direct()
                mode = "direct"
            elif self._graph is not None:
                self._graph.replay()
                mode = "graph"
            else:
                self._body()
                mode = "captured"
            e1.record(st.stream)
        st.stream.synchronize()
        ms = e0.elapsed_time(e1)
        if st.cap is None:
            S, Y, crossings = unpack_fit_sums(st.sums.cpu().numpy())
        else:
            if int(st.maxk.item()) > st.cap.x.capacity:
                raise RuntimeError(f"crossing records overflowed: {int(st.maxk.item())} > {st.cap.x.capacity}")
            S = st.S[:, :self.I].cpu().numpy()
            Y = st.Y[:, :self.I].cpu().numpy()
            crossings = st.crossings[:self.I].cpu().numpy()
        gvn = st.gv[:self.I].cpu().numpy()
        if graph and self._graph is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=st.stream):
                self._body()
            self._graph = g
        fix, tunes, good = fit_one_turn(S, Y)
        fix = fix * st.unit
        new = gvn + fix
        dr = np.where(good, fix[:, 0], 0.0)
        # back to p-format orbit parameters at azimuth 0 (vphi from the speed)
        vtot = self.conv.Ek2v(self.E)
        for i in np.nonzero(good)[0]:
            vr, vz = new[i, 1], new[i, 3]
            vf = math.sqrt(max(vtot[i] ** 2 - vr * vr - vz * vz, 0.0))
            self.r[i], self.z[i] = new[i, 0], new[i, 2]
            self.pr[i], self.pz[i] = math.atan2(vr, vf), math.atan2(vz, vf)
        rec_ = {"ms": ms, "launches": st.launches, "mode": mode, "particle_turns": float(crossings.sum()),
                "max_abs_dr": float(np.abs(dr).max()), "dr": dr, "tunes": tunes, "good": good,
                "crossings": crossings}
        self.history.append(rec_)
        return rec_

    def run(self, iterations=3, tol=1e-6, graph=True):
        """Iterates until the largest orbit change is below `tol` [m]."""
        for _ in range(iterations):
            rec = self.iterate(graph)
            if rec["max_abs_dr"] < tol:
                break
        return self.history[-1]

    def padding(self, block=32):
        """Launch slots per particle: the push kernel's blocks over the whole bunch."""
        return math.ceil(self.N / block) * block / self.N
