"""The tracking loop on the GPU.

FFAG_RungeKutta mirrors the reference's integrator object
(src/FFAG_track.py:31-1049): the two bunch-tracking loops
rk4_solve_dt_bunch3_withSC_boris / rk4_solve_dt_bunch3_withSC keep their
signatures and per-step semantics (injection, space-charge cadence and
extrapolation, push, dumps, the stop test every 1000 steps), and Boris_solve /
rk4_step_malloc are kept as drop-in single-step calls on an N x 16 matrix.

Design: everything that depends only on the step index (the time sequence
t_{s+1} = t_s + dt, the RF frequency/voltage per step, each particle's
injection step, the dump steps) is computed on the host once per chunk of
steps, so one fused kernel launch can advance the bunch through every step
up to the next event (space-charge update, dump, stop test).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from .bunch import FFAG_Bunch
from .constants import C_LIGHT, COLUMNS, FFAG_ConversionTools, FFAG_GlobalParameters
from .dump import PositionDump

TABLE_CHUNK = 1 << 16


class StepClock:
    """Times and per-step RF scalars for absolute steps [0, n), extended in
    chunks.  t[s] is the start time of step s, built by the same repeated
    float64 addition as the reference loop (t_PreStep = t_PreStep + step_t)."""

    def __init__(self, t_start: float, dt: float, emap, solver: str, device):
        self.t0 = float(t_start)
        self.dt = float(dt)
        self.emap = emap
        self.solver = solver
        self.device = device
        self.t = np.array([self.t0], dtype=np.float64)  # t[0..n]
        self.n = 0
        self.drf = None
        self.acc = None

    def ensure(self, nsteps: int) -> bool:
        """Makes tables cover steps [0, nsteps).  Returns True if extended."""
        if nsteps <= self.n:
            return False
        new_n = max(nsteps, self.n + TABLE_CHUNK)
        add = new_n - self.n
        ext = np.empty(add + 1, dtype=np.float64)
        ext[0] = self.t[-1]
        ext[1:] = self.dt
        ts = np.add.accumulate(ext)  # sequential sums: t_{s+1} = t_s + dt
        self.t = np.concatenate([self.t, ts[1:]])
        self.n = new_n
        self._build_tables()
        return True

    def _build_tables(self):
        import torch
        em = self.emap
        tp = self.t[: self.n]
        if self.solver == "Boris":
            f, v = em.Interpolation1D_freq_curve(tp)
            drf = f * np.pi * 2 * self.dt
            acc = em.acc_Etot_uniform * v
        else:
            h = self.dt
            ts = np.stack([tp, tp + 0.5 * h, tp + 0.5 * h, tp + h], axis=1).reshape(-1)
            f, v = em.Interpolation1D_freq_curve(ts)
            drf = f * np.pi * 2
            acc = em.acc_Etot_uniform * v
        self.drf = torch.from_numpy(np.ascontiguousarray(drf)).to(self.device)
        self.acc = torch.from_numpy(np.ascontiguousarray(acc)).to(self.device)
        self.table = _lib.StepTable()
        self.table.drf = self.drf.data_ptr()
        self.table.acc = self.acc.data_ptr()
        self.table.nsteps = self.n

    def windows(self, s0: int, s1: int):
        """Injection windows [(t - dt) * 1e9, t * 1e9] of steps s0..s1-1."""
        t = self.t[s0:s1]
        return (t - self.dt) * 1e9, t * 1e9


def _aperture(gp) -> "_lib.Aperture":
    ap = _lib.Aperture()
    if getattr(gp, "Aperture_enable", False) and gp.Aperture_m is not None:
        ap.enable = 1
        ap.rmin, ap.rmax, ap.zmin, ap.zmax = (float(x) for x in gp.Aperture_m)
    return ap


def _consts(gp) -> "_lib.Consts":
    cs = _lib.Consts()
    cs.q, cs.c, cs.m0, cs.E0 = float(gp.q), float(gp.c), float(gp.m0), float(gp.E0)
    return cs


def _part1by3(x):
    """The 15 low bits of each int64 of x spread to every fourth bit."""
    x = x & 0x7FFF
    x = (x | (x << 24)) & 0x000000FF000000FF
    x = (x | (x << 12)) & 0x000F000F000F000F
    x = (x | (x << 6)) & 0x0303030303030303
    x = (x | (x << 3)) & 0x1111111111111111
    return x


def morton_order(cols, start: int, n: int, period: float):
    """A thread-to-particle permutation (int32, device) of particles
    [start, start + n) in Morton (Z-curve) order of (r, vr, azimuth within
    the sector, f5), each quantised to 15 bits over the range's span:
    particles with nearby keys sit near each other in the coordinates that
    pick the z-Taylor nodes of the next steps.  Non-finite values count as
    the span's low end.  Particles not in flight (not injected, or lost: the
    push kernels take a different branch for them) come after all particles
    in flight, so that warps do not mix the two branches."""
    import torch
    sl = slice(start, start + n)
    x = torch.stack([cols["r"][sl], cols["vr"][sl], torch.remainder(cols["fi"][sl], period), cols["f5"][sl]])
    x = torch.nan_to_num(x, nan=0.0, posinf=0.0, neginf=0.0)
    lo = x.amin(1, keepdim=True)
    span = (x.amax(1, keepdim=True) - lo).clamp_min(1e-300)
    q = ((x - lo) / span * 32767.0).to(torch.int64).clamp_(0, 32767)
    key = _part1by3(q[0]) | (_part1by3(q[1]) << 1) | (_part1by3(q[2]) << 2) | (_part1by3(q[3]) << 3)
    if "inj" in cols and "surv" in cols:
        idle = (cols["inj"][sl] != 1) | (cols["surv"][sl] != 1)
        key |= idle.to(torch.int64) << 61
    return torch.argsort(key).to(torch.int32)


class Pusher:
    """Binds a bunch to the field / RF / aperture descriptors and launches
    fused push kernels.

    order: "morton" -- each launch's threads take the particles in the
    Morton order of morton_order, computed on the launch's stream for every
    particle range pushed and recomputed every `order_every` launches of
    that range (0: never), so that a warp's z-Taylor node loads share cache
    lines; None -- thread t advances particle t; "auto" (default) -- morton
    for the float64 pushers, whose time goes to those loads (c1 Boris: 2.64
    -> 2.47 ms per 1e5-particle turn; 1e6 particles: 23.9 -> 18.7 ms), None
    for the float32-field ones (no gain measured).  The results are the same
    either way.  Ranges under `order_min` particles keep the identity."""

    def __init__(self, bunch: FFAG_Bunch, gp, solver: str, precision: str = "fp64", order="auto",
                 order_every: int = 64, order_min: int = 4096):
        import torch
        if order not in ("morton", None, "auto"):
            raise ValueError(f"order must be 'morton', 'auto' or None, not {order!r}")
        if order == "auto":
            order = "morton" if precision == "fp64" else None
        self.order = order
        self.order_every = int(order_every)
        self.order_min = int(order_min)
        self._orders = {}
        self._soa_views = {}
        self.bunch = bunch
        self.gp = gp
        self.solver = solver
        self.fm = gp.Bmap.device_map(bunch.device)
        self.rf = gp.Emap.rf_desc(device=bunch.device)
        self.ap = _aperture(gp)
        self.cs = _consts(gp)
        # field-error harmonics (FFAG_BField_Error): carried by the device map
        # and set on it before each push, since maps are shared between pushers
        self.harmonics = getattr(gp, "BHarmonics", None)
        self.flags = _lib.FFA_RK4 if solver == "RK4" else _lib.FFA_BORIS
        if precision in ("fp32c", "fp32"):
            if solver == "RK4" and precision == "fp32":
                raise NotImplementedError("the float32 push is Boris-only (RK4 takes fp64 or fp32c)")
            self.flags |= _lib.FFA_FP32C if precision == "fp32c" else _lib.FFA_FP32
        elif precision != "fp64":
            raise ValueError(f"precision must be fp64, fp32c or fp32, not {precision!r}")
        if getattr(gp.Emap, "physical_sum", False):
            self.flags |= _lib.FFA_RF_PHYSICAL_SUM
        self.stream = torch.cuda.current_stream(bunch.device)
        # launch shape (threads-per-block index, register-cap index) of the
        # Boris kernels; (0, 0) is the default, autotune.tune_push picks others
        self.shape = (0, 0)

    def push(self, clock: StepClock, step0: int, nsteps: int, sc_step: int = 0, xing=None, start: int = 0,
             count=None, stream=None) -> None:
        """Advances particles [start, start + count) (default: all) by nsteps
        steps from absolute step step0 on `stream` (default: the pusher's)."""
        L = _lib.lib()
        b = self.bunch
        flags = self.flags | _lib.shape_flags(*self.shape)
        n = b.n - start if count is None else count
        if start < 0 or n < 0 or start + n > b.n:
            raise ValueError(f"particle range [{start}, {start + n}) outside the bunch of {b.n}")
        soa = b.soa() if start == 0 else self._soa_at(b.soa(), start)
        self.fm.set_harmonics(self.harmonics)
        st = self.stream if stream is None else stream
        s = st.cuda_stream
        if self.order is not None and n >= self.order_min and hasattr(b, "cols"):
            soa = _lib.StateSoA.from_buffer_copy(soa)
            soa.order = self._order_for(start, n, st).data_ptr()
        args = (self.fm.handle, ctypes.byref(self.rf), ctypes.byref(self.ap), ctypes.byref(self.cs),
                ctypes.byref(clock.table), ctypes.byref(soa), n, step0, nsteps, clock.dt,
                sc_step, flags, s, b.status.data_ptr())
        if xing is None:
            _lib.check(L.ffa_push(*args), "ffa_push")
        else:
            _lib.check(L.ffa_push_crossing(*args, ctypes.byref(xing)), "ffa_push_crossing")


    def _soa_at(self, base, start):
        """The SoA view of particles start.. (cached: the bunch's columns do
        not move while it lives)."""
        key = (start, base.r)
        v = self._soa_views.get(key)
        if v is None:
            v = self._soa_views[key] = _lib.soa_offset(base, start)
        return v

    def _order_for(self, start, n, stream):
        """The Morton permutation of particles [start, start + n), made on
        `stream` (where the launch that reads it runs) when missing or
        `order_every` launches old."""
        import torch
        ent = self._orders.get((start, n))
        if ent is None or (self.order_every > 0 and ent[1] >= self.order_every):
            period = 2 * np.pi / float(getattr(self.gp.Bmap, "Nsectors", 1) or 1)
            with torch.cuda.stream(stream):
                ent = [morton_order(self.bunch.cols, start, n, period), 0]
            self._orders[(start, n)] = ent
        ent[1] += 1
        return ent[0]


class CrossingCapture:
    """Device buffers of the azimuth-crossing records for a set of target
    azimuths, and their conversion to the post-step rows the reference's
    PositionDumpBunch appends (src/FFAG_dump.py:1098-1130).

    A launch of `nsteps` steps can see a particle cross one target at most
    1 + nsteps * dt * f_max / (2 pi) times, with f_max = c / r_low the
    fastest angular velocity inside the aperture (or the field map); the
    capacity is sized from that bound and an overflow raises."""

    def __init__(self, bunch: FFAG_Bunch, targets, gp, dt: float):
        import torch
        if not 1 <= len(targets) <= _lib.MAX_CROSSING_TARGETS:
            raise ValueError(f"1 to {_lib.MAX_CROSSING_TARGETS} crossing targets per bunch")
        self.bunch = bunch
        self.dt = dt
        self.x = _lib.Crossing()
        self.x.ntargets = len(targets)
        for k, t in enumerate(targets):
            self.x.target[k] = float(t) % (2 * np.pi)
        r_low = gp.Aperture_m[0] if getattr(gp, "Aperture_enable", False) else gp.Bmap.r_min
        self.f_max = C_LIGHT / max(float(r_low), 1e-3)
        self.count = torch.zeros(1, dtype=torch.int64, device=bunch.device)
        self.buf = torch.empty(0, dtype=torch.float64, device=bunch.device)

    def max_steps(self) -> int:
        """Longest launch whose bound stays at 5 records per particle and target."""
        return max(1, int(3 * 2 * np.pi / (self.dt * self.f_max)))

    def prepare(self, nsteps: int):
        import torch
        per = 2 + int(np.ceil(nsteps * self.dt * self.f_max / (2 * np.pi)))
        cap = self.bunch.n * self.x.ntargets * per
        if self.buf.numel() < cap * _lib.CROSSING_RECORD:
            self.buf = torch.empty(cap * _lib.CROSSING_RECORD, dtype=torch.float64, device=self.bunch.device)
        self.count.zero_()
        self.x.buf = self.buf.data_ptr()
        self.x.capacity = cap
        self.x.count = self.count.data_ptr()
        return self.x

    def records(self) -> np.ndarray:
        """The launch's records, sorted by (target, step, particle)."""
        k = int(self.count.item())
        if k > self.x.capacity:
            raise RuntimeError(f"crossing records overflowed: {k} > {self.x.capacity}")
        rec = self.buf[:k * _lib.CROSSING_RECORD].view(k, _lib.CROSSING_RECORD).cpu().numpy()
        return rec[np.lexsort((rec[:, 1], rec[:, 2], rec[:, 0]))]

    def rows(self, rec: np.ndarray) -> np.ndarray:
        return crossing_rows(rec, self.bunch._host_static)


def crossing_rows(rec: np.ndarray, host_static: np.ndarray) -> np.ndarray:
    """Post-step v-format rows (N x 16) of crossing records: the LocalBunch
    rows PositionDumpBunch.check_and_dump selects (src/FFAG_dump.py:1120);
    injection time and the ID columns come from the bunch's host matrix."""
    idx = rec[:, 1].astype(np.int64)
    out = np.zeros((rec.shape[0], 16))
    out[:, 0:6] = rec[:, 11:17]
    out[:, 6] = host_static[idx, COLUMNS["inj_t"]]
    out[:, 7] = rec[:, 19]
    out[:, 8] = rec[:, 18]
    out[:, 9] = rec[:, 17]
    out[:, 10:13] = rec[:, 20:23]
    out[:, 13:16] = host_static[idx, 13:16]
    return out


class StepDumpSchedule:
    """Steps at which a StepDumpBunch fires: start < t_post < end and the
    interval index floor((t - start) / interval) changes between t_pre and
    t_post (StepDumpBunch.check_and_dump, src/FFAG_dump.py:330-356)."""

    def __init__(self, dump):
        self.dump = dump

    def steps_in(self, t_pre: np.ndarray, t_post: np.ndarray) -> np.ndarray:
        d = self.dump
        inside = (d.start_time < t_post) & (t_post < d.end_time)
        a = np.floor_divide(t_pre - d.start_time, d.time_interval)
        b = np.floor_divide(t_post - d.start_time, d.time_interval)
        return np.nonzero(inside & (a != b))[0]


class FFAG_RungeKutta:
    """Bunch trackers (src/FFAG_track.py:31-1049)."""

    def __init__(self, precision: str = "fp64", verbose: bool = True):
        self.running = True
        self.precision = precision
        self.verbose = verbose
        self.last_run = {}

    # ------------------------------------------------ drop-in single steps
    def Boris_solve(self, t, mat_in, dt, *scratch, GlobalParameters=None):
        """One Boris step of the N x 16 Boris v-format matrix `mat_in`, in
        place (src/FFAG_track.py:948-1049).  The reference's 25 scratch
        arrays are accepted and ignored; GlobalParameters may be passed
        positionally last, as the reference does."""
        if GlobalParameters is None:
            GlobalParameters = scratch[-1]
        out = single_step(mat_in, float(t), float(dt), GlobalParameters, "Boris", self.precision)
        mat_in[...] = out
        return mat_in

    def rk4_step_malloc(self, func, t, r, h, GlobalParameters, *scratch):
        """One RK4 step of the N x 16 RK4 v-format matrix; returns the
        increment like the reference (src/FFAG_track.py:51-61), plus the
        three field arrays it returned (not computed here: None)."""
        new = single_step(r, float(t), float(h), GlobalParameters, "RK4", "fp64")
        return new - np.asarray(r), None, None, None

    # ---------------------------------------------------------- the loops
    def rk4_solve_dt_bunch3_withSC_boris(self, func, t_start, BunchObj, GlobalParameters, LocalParameters):
        return self._solve("Boris", t_start, BunchObj, GlobalParameters, LocalParameters)

    def rk4_solve_dt_bunch3_withSC(self, func, t_start, BunchObj, GlobalParameters, LocalParameters):
        return self._solve("RK4", t_start, BunchObj, GlobalParameters, LocalParameters)

    def _solve(self, solver, t_start, b: FFAG_Bunch, gp, lp):
        import torch
        stop = lp["stop_condition"]
        dt = float(lp["time_step"])
        enable_sc = bool(lp.get("enable_SC", False))
        sc_type = lp.get("SC_type", 1)
        SC_step = int(lp.get("SC_step", 1))
        dumps = lp.get("step_dumps")
        comm = lp.get("comm")
        max_stepsN = int(stop["max_stepsN"])
        max_fi = stop["max_turn"] * np.pi * 2
        max_time = stop["max_time"]
        if b.BunchType != solver:
            raise ValueError(f"bunch type {b.BunchType} does not match the {solver} solver")
        if enable_sc and sc_type != 1:
            raise NotImplementedError("only the 2.5D slice-by-slice space charge (SC_type 1) is built")

        pusher = Pusher(b, gp, solver, self.precision)
        clock = StepClock(t_start, dt, gp.Emap, solver, b.device)
        sc = None
        if enable_sc:
            from .space_charge import SpaceCharge
            sc = SpaceCharge(b, hockney=bool(lp.get("SC_hockney", False)))
        dump_sched = [StepDumpSchedule(d) for d in (dumps.step_dumps() if dumps is not None else [])]
        pdumps = dumps.particle_step_dumps() if dumps is not None else []
        pos_dumps = dumps.position_dumps() if dumps is not None else []
        xcap = CrossingCapture(b, [d.target_azimuth_angle for d in pos_dumps], gp, dt) if pos_dumps else None

        steps_i = 0
        sched_end = 0
        fi_sum = torch.zeros(1, dtype=torch.float64, device=b.device)
        fi_cnt = torch.zeros(1, dtype=torch.int64, device=b.device)
        t_wall = time.time()
        n_launch = 0
        b.reset_schedule_count()
        while steps_i < max_stepsN:
            if clock.ensure(steps_i + 1) or steps_i >= sched_end:
                clock.ensure(steps_i + 1)
                lo, hi = clock.windows(steps_i, clock.n)
                b.set_injection_schedule(lo, hi, steps_i)
                b.reset_schedule_count()
                sched_end = clock.n
            # the next event bounds the fused chunk
            end = min(max_stepsN, (steps_i // 1000 + 1) * 1000, sched_end)
            if enable_sc:
                if steps_i % SC_step == 0:
                    _lib.check(_lib.lib().ffa_inject(ctypes.byref(b.soa()), b.n, steps_i, pusher.stream.cuda_stream),
                               "ffa_inject")
                    sc.update(first=(steps_i == 0))
                end = min(end, (steps_i // SC_step + 1) * SC_step)
            dump_at = None
            for ds in dump_sched:
                hit = ds.steps_in(clock.t[steps_i:end], clock.t[steps_i + 1:end + 1])
                if hit.size:
                    cand = steps_i + int(hit[0])
                    dump_at = cand if dump_at is None else min(dump_at, cand)
            for pd in pdumps:
                if pd.save_flag:
                    continue
                hit = np.nonzero(pd.fires(clock.t[steps_i:end], clock.t[steps_i + 1:end + 1]))[0]
                if hit.size:
                    cand = steps_i + int(hit[0])
                    dump_at = cand if dump_at is None else min(dump_at, cand)
            if dump_at is not None:
                end = dump_at + 1
            pre_alive = None
            if pdumps and dump_at is not None and any(
                    not pd.save_flag and pd.fires(clock.t[dump_at], clock.t[dump_at + 1]) for pd in pdumps):
                # the trigger step alone, so its pre-step survival can be read
                if dump_at > steps_i:
                    end = dump_at
                    dump_at = None
                else:
                    pre_alive = b.alive_at_step(steps_i)
            t_chunk = clock.t[steps_i + 1:end + 1]
            capture = xcap is not None and any(not d.save_flag and d.in_window(t_chunk).any() for d in pos_dumps)
            if capture and end - steps_i > xcap.max_steps():
                end = steps_i + xcap.max_steps()
                t_chunk = clock.t[steps_i + 1:end + 1]
            pusher.push(clock, steps_i, end - steps_i, SC_step if enable_sc else 0,
                        xcap.prepare(end - steps_i) if capture else None)
            n_launch += 1
            if capture:
                rec = xcap.records()
                for k, d in enumerate(pos_dumps):
                    r = rec[rec[:, 0] == k]
                    tp = clock.t[r[:, 2].astype(np.int64) + 1]
                    keep = d.in_window(tp) if not d.save_flag else np.zeros(len(r), bool)
                    if keep.any():
                        if isinstance(d, PositionDump):
                            d.add_particles(xcap.rows(r[keep]), tp[keep], solver)
                        else:
                            d.add_particles(xcap.rows(r[keep]), tp[keep])
                            d.add_records(r[keep], tp[keep])
            for d in pos_dumps:
                if not d.save_flag and (t_chunk > d.end_time).any():
                    d.save_all_particles(solver)
                    d.save_flag = True
            steps_i = end
            if dump_at is not None:
                t_post = clock.t[steps_i]
                t_pre = clock.t[steps_i - 1]
                for ds in dump_sched:
                    if ds.steps_in(np.array([t_pre]), np.array([t_post])).size:
                        ds.dump.dump_bunch(b, t_post, data_type=solver)
                if pre_alive is not None:
                    local = b.LocalBunch
                    for pd in pdumps:
                        if not pd.save_flag and pd.fires(t_pre, t_post):
                            rows = np.nonzero(np.isin(local[:, 15].astype(np.int64), pd.tracked_global_ids))[0]
                            pd.record(local[rows], pre_alive[rows], t_post, solver)
            for pd in pdumps:
                if not pd.save_flag and clock.t[steps_i - 1] > pd.end_time:
                    pd.dump_all_particles()
                    pd.save_flag = True
            if steps_i % 1000 == 0:
                b.UpdateParticleNumGlobal(comm)
                _lib.check(_lib.lib().ffa_mean_fi(ctypes.byref(b.soa()), b.n, fi_sum.data_ptr(), fi_cnt.data_ptr(),
                                                  pusher.stream.cuda_stream), "ffa_mean_fi")
                s, c = float(fi_sum.item()), int(fi_cnt.item())
                if comm is not None:
                    v = torch.tensor([s, float(c)], dtype=torch.float64)
                    comm.all_reduce(v)
                    s, c = float(v[0]), int(v[1])
                mean_fi = s / c if c > 0 else float("nan")
                t_now = clock.t[steps_i]
                if self.verbose and (comm is None or comm.get_rank() == 0):
                    print(f"current step={steps_i:.0f}, turn ~= {mean_fi / np.pi / 2:.2f}, "
                          f"remain particles: {b.SurvivedNum}. tracking time: {t_now * 1e6:.2f} us, "
                          f"clock: {time.strftime('%m-%d %H:%M:%S', time.localtime())}", flush=True)
                if abs(mean_fi) > max_fi:
                    break
                if t_now > max_time:
                    break
        torch.cuda.synchronize(b.device)
        self.last_run = {"steps": steps_i, "t_end": float(clock.t[steps_i]), "launches": n_launch,
                         "wall_s": time.time() - t_wall, "status": b.status_counts()}
        return 0


def single_step(mat, t, dt, gp, solver, precision="fp64"):
    """Advances an N x 16 v-format matrix by one step on the GPU and returns
    the new matrix (cols 6, 13-15 copied through)."""
    import torch
    a = np.ascontiguousarray(np.asarray(mat, dtype=np.float64))
    n = a.shape[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    b = _EphemeralBunch(a, solver, dev)
    clock = StepClock(t, dt, gp.Emap, solver, dev)
    clock.ensure(1)
    pusher = Pusher(b, gp, solver, precision)
    pusher.push(clock, 0, 1, 0)
    out = b.matrix()
    return out


class _EphemeralBunch:
    """Device SoA for one N x 16 matrix without the injection bookkeeping
    (the reference's Boris_solve takes the flags as they are)."""

    def __init__(self, a, solver, dev):
        import torch
        self.BunchType = solver
        self.device = dev
        self.n = a.shape[0]
        self._a = a
        self.aos = a.to(dev, torch.float64).contiguous() if torch.is_tensor(a) else torch.from_numpy(a).to(dev)
        f64 = dict(dtype=torch.float64, device=dev)
        self.cols = {k: torch.empty(self.n, **f64) for k in ("r", "vr", "z", "vz", "fi", "f5", "rf",
                                                             "esc_r", "esc_z", "esc_fi")}
        self.cols["inj"] = torch.empty(self.n, dtype=torch.uint8, device=dev)
        self.cols["surv"] = torch.empty(self.n, dtype=torch.uint8, device=dev)
        self.status = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int64, device=dev)
        s = _lib.StateSoA()
        for name, _ in _lib.StateSoA._fields_:
            t = self.cols.get(name)
            setattr(s, name, t.data_ptr() if t is not None else None)
        self._soa = s
        _lib.check(_lib.lib().ffa_aos_to_soa(self.aos.data_ptr(), self.n, ctypes.byref(s), _lib.stream_ptr(None)),
                   "ffa_aos_to_soa")

    def soa(self):
        return self._soa

    def matrix(self):
        _lib.check(_lib.lib().ffa_soa_to_aos(ctypes.byref(self._soa), self.n, self.aos.data_ptr(), _lib.stream_ptr(None)),
                   "ffa_soa_to_aos")
        return self.aos.cpu().numpy()


def split_spans(n: int, chunks: int) -> list:
    """[start, end) ranges that cover 0..n in order: every start a multiple
    of 32 (edges rounded down to whole warps, the last range taking the
    remainder, so sizes differ by less than 64), no empty range, at most
    `chunks` of them (fewer when n has fewer warps)."""
    k = max(1, min(int(chunks), max(1, n // 32)))
    edges = [0] + [((n * c) // k) // 32 * 32 for c in range(1, k)] + [n]
    return [(a, e) for a, e in zip(edges[:-1], edges[1:]) if e > a]


class MatrixTracker:
    """Host-buffer entry point: advances an N x 16 v-format matrix that lives
    in host memory by `nsteps` fused steps and writes the result back (the
    call a host-side caller of Boris_solve / rk4_step makes, batched over
    steps).  Device buffers are allocated once; each call copies the matrix
    in, converts it to SoA, pushes, converts back and copies it out.

    chunks > 1 splits the bunch into that many particle ranges (multiples of
    32), each on its own stream: one range's host copies overlap another's
    push, and the pushes of all ranges are resident together, so the push
    itself is not slowed.  Every particle sees the same arithmetic either
    way."""

    def __init__(self, n, gp, solver="Boris", precision="fp64", device=None, chunks=2):
        import torch
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.n = n
        self.gp = gp
        self.solver = solver
        self.precision = precision
        self.b = _EphemeralBunch(np.zeros((n, 16)), solver, self.dev)
        self.pusher = Pusher(self.b, gp, solver, precision)
        self.clock = None
        self.launches = 0
        self.spans = split_spans(n, chunks)
        self.streams = [torch.cuda.Stream(self.dev) for _ in self.spans] if len(self.spans) > 1 else []
        self._soas = [_lib.soa_offset(self.b.soa(), a) for a, _ in self.spans]
        self._ready = torch.cuda.Event()
        self._done = [torch.cuda.Event() for _ in self.spans]

    def bind_clock(self, t_start, dt, nsteps_total):
        self.clock = StepClock(t_start, dt, self.gp.Emap, self.solver, self.dev)
        self.clock.ensure(nsteps_total)

    def run(self, host_in, host_out, step0, nsteps):
        """host_in / host_out: pinned (or pageable) float64 torch tensors (n, 16).
        The work is ordered after what the pusher's stream holds, and that
        stream waits for it (synchronise it to read host_out)."""
        import torch
        L = _lib.lib()
        b = self.b
        main = self.pusher.stream
        if not self.streams:
            s = main.cuda_stream
            b.aos.copy_(host_in, non_blocking=True)
            _lib.check(L.ffa_aos_to_soa(b.aos.data_ptr(), b.n, ctypes.byref(b.soa()), s), "ffa_aos_to_soa")
            self.pusher.push(self.clock, step0, nsteps, 0)
            _lib.check(L.ffa_soa_to_aos(ctypes.byref(b.soa()), b.n, b.aos.data_ptr(), s), "ffa_soa_to_aos")
            host_out.copy_(b.aos, non_blocking=True)
            self.launches += 3
            return
        ready = self._ready
        ready.record(main)
        row = b.aos.stride(0) * b.aos.element_size()
        for (a, e), st, soa, done in zip(self.spans, self.streams, self._soas, self._done):
            st.wait_event(ready)
            with torch.cuda.stream(st):
                b.aos[a:e].copy_(host_in[a:e], non_blocking=True)
                _lib.check(L.ffa_aos_to_soa(b.aos.data_ptr() + a * row, e - a, ctypes.byref(soa), st.cuda_stream),
                           "ffa_aos_to_soa")
                self.pusher.push(self.clock, step0, nsteps, 0, start=a, count=e - a, stream=st)
                _lib.check(L.ffa_soa_to_aos(ctypes.byref(soa), e - a, b.aos.data_ptr() + a * row, st.cuda_stream),
                           "ffa_soa_to_aos")
                host_out[a:e].copy_(b.aos[a:e], non_blocking=True)
            done.record(st)
            main.wait_event(done)
            self.launches += 3
