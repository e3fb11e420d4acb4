"""Learned one-sector transfer map: a residual MLP on the tensor cores.

PyFFA (the reference) tracks every particle through every step with its
pushers.  For long tracking at fixed energy, this module replaces the
tracker between sector entrances with a learned map of one sector, trained
on crossings that the plain azimuth-domain tracker produces, and keeps the
plain tracker as the arbiter:

- the plain pusher here is the FP64 azimuth-domain RK4 tracker
  (ffa_theta_track; FunctionForSEO, src/FFAG_track.py:1597-1640, with
  rk4_solve stage azimuths, src/FFAG_track.py:582-611), S steps per sector;
- coordinates at the sector entrance (azimuth 0 of every sector) are taken
  relative to the closed orbit of the particle's energy and scaled to
  Floquet (Twiss-normalised) coordinates, so that the training domain
  "amplitudes up to A_x / A_p" is the unit disc in each transverse plane:
  s = (u, pu, v, pv, e) with e the energy mapped to [-1, 1];
- the network (ffa_mlp_*; widths 6 -> 256 -> 256 -> 256 -> 6, SiLU, bfloat16
  operands with float32 accumulation, a float32 skip connection of first
  and second order) maps s at one sector entrance to s at the next; the skip
  connection is the least-squares second-order map, the MLP learns what it
  misses (the third and higher orders);
- tracking applies the map K times per launch on float32 states; states
  outside the domain go to the plain tracker for the rest of the run, and
  every `audit_every` turns a random `audit_frac` of the learned states is
  tracked one sector by both; a state whose map error exceeds `audit_tol`
  goes to the plain tracker too.

The error measure of a state is the largest of |dr| / r_co, |dpr|, |dz| / r_co,
|dpz| (pr, pz are p_r / p, p_z / p): coordinates relative to the machine
scale.

Everything runs on one GPU; torch tensors carry device memory and the
float64 coordinate transforms.  There is no CPU path: without
libffa_cuda.so every call raises.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _lib
from .constants import FFAG_ConversionTools

HIDDEN = _lib.MLP_HIDDEN
N_PARAMS = _lib.MLP_PARAMS
LOSS_PARTS = 148


def _layout():
    shapes = [("W1", (16, 256)), ("b1", (256,)), ("W2", (256, 256)), ("b2", (256,)), ("W3", (256, 256)),
              ("b3", (256,)), ("W4", (256, 8)), ("b4", (8,)), ("Ws", (8, 8)), ("bs", (8,)), ("Wq", (16, 8))]
    out, o = {}, 0
    for k, sh in shapes:
        out[k] = (o, sh)
        o += int(np.prod(sh))
    assert o == N_PARAMS
    return out


LAYOUT = _layout()
# the used part of each padded block (6 inputs, 6 outputs)
USED = {"W1": (6, 256), "b1": (256,), "W2": (256, 256), "b2": (256,), "W3": (256, 256), "b3": (256,),
        "W4": (256, 6), "b4": (6,), "Ws": (6, 6), "bs": (6,), "Wq": (15, 6)}
# the quadratic skip features s_i s_j, i <= j < 5, in the kernels' order
QUAD = [(i, j) for i in range(5) for j in range(i, 5)]
SKIP = ("Ws", "bs", "Wq")


def block(p, name):
    """View of one parameter block of a flat parameter vector (numpy or torch)."""
    o, sh = LAYOUT[name]
    return p[o:o + int(np.prod(sh))].reshape(sh)


def init_params(seed=0):
    """Flat float32 parameters: scaled normal hidden weights, zero output
    layer, biases and skip layer (the network starts as the identity map)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(N_PARAMS, np.float32)
    block(p, "W1")[:6] = rng.standard_normal((6, HIDDEN)) * (1.0 / math.sqrt(6.0)) * 1.5
    block(p, "W2")[:] = rng.standard_normal((HIDDEN, HIDDEN)) * math.sqrt(2.0 / HIDDEN)
    block(p, "W3")[:] = rng.standard_normal((HIDDEN, HIDDEN)) * math.sqrt(2.0 / HIDDEN)
    return p


def to_dict(p):
    """float64 dict of the used blocks (the oracle's parameter format)."""
    p = np.asarray(p, np.float32)
    return {k: block(p, k)[tuple(slice(0, s) for s in sh)].astype(np.float64) for k, sh in USED.items()}


def from_dict(d):
    p = np.zeros(N_PARAMS, np.float32)
    for k, sh in USED.items():
        block(p, k)[tuple(slice(0, s) for s in sh)] = np.asarray(d[k], np.float32)
    return p


def _torch():
    import torch
    return torch


# ------------------------------------------------------------- the plain tracker
class SectorTracker:
    """Whole sectors of the azimuth-domain RK4 tracker (ffa_theta_track) on
    device tensors: x0 (m, 5) = r, pr, z, pz, P -> (m, 4)."""

    def __init__(self, bmap, q, steps_per_sector=256, device=None):
        torch = _torch()
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.fm = bmap.device_map(self.dev)
        self.q = float(q)
        self.nsectors = int(bmap.Nsectors)
        self.period = 2 * np.pi / self.nsectors
        self.S = int(steps_per_sector)
        self.launches = 0

    def run(self, x0, n_sectors=1):
        torch = _torch()
        x0 = x0.to(self.dev, torch.float64).contiguous()
        m = x0.shape[0]
        x1 = torch.empty((m, 4), dtype=torch.float64, device=self.dev)
        if m == 0 or n_sectors == 0:
            x1.copy_(x0[:, :4])
            return x1
        d = _lib.ThetaTrackDesc()
        d.m, d.n_points, d.time_mode = m, int(n_sectors) * self.S + 1, 0
        d.traj_cols, d.t_end, d.q = 2, float(n_sectors) * self.period, self.q
        d.x0, d.x1, d.traj = x0.data_ptr(), x1.data_ptr(), None
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        _lib.check(_lib.lib().ffa_theta_track(self.fm.handle, ctypes.byref(d), stream), "ffa_theta_track")
        self.launches += 1
        return x1


class TimeDomainSectorTracker:
    """Whole sectors of the time-domain Boris pusher -- the tracking loop's
    own plain pusher, the compensated float32 one by default -- behind
    SectorTracker's interface: x0 (m, 5) = r, pr, z, pz, P at a sector
    entrance -> (m, 4) at the entrance n_sectors later.  The lattice repeats
    every sector, so every state starts at azimuth 0; all states are pushed
    in one launch of steps dt (RF off, no aperture) until each azimuth has
    passed n_sectors sector angles, the push kernels capture the crossing
    step, and the state at that azimuth comes from a cubic Hermite
    interpolation of the step in Cartesian coordinates
    (coscan.crossing_states); pr, pz = vr / v, vz / v with the speed v of the
    state's momentum (a static magnetic field keeps it).  gp: the lattice's
    FFAG_GlobalParameters (its Bmap is used); chunk: states per launch."""

    def __init__(self, gp, dt, precision="fp32c", device=None, chunk=1 << 21):
        import os
        import tempfile
        torch = _torch()
        from . import synthetic
        from .constants import FFAG_GlobalParameters
        from .fields import FFAG_EField_new
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.gp = FFAG_GlobalParameters()
        self.gp.AddBMap(gp.Bmap)
        self.gp.AddEMap(FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")),
                                        EnableFlag=False))
        self.dt = float(dt)
        self.precision = precision
        self.nsectors = int(gp.Bmap.Nsectors)
        self.period = 2 * np.pi / self.nsectors
        self.chunk = int(chunk)
        self.q = float(self.gp.q)
        self.launches = 0
        self._clock = None

    def _clock_for(self, nsteps):
        from .track import StepClock
        if self._clock is None:
            self._clock = StepClock(0.0, self.dt, self.gp.Emap, "Boris", self.dev)
        self._clock.ensure(nsteps + 1)
        return self._clock

    def run(self, x0, n_sectors=1):
        torch = _torch()
        x0 = x0.to(self.dev, torch.float64).contiguous()
        m = x0.shape[0]
        if m == 0 or n_sectors == 0:
            return x0[:, :4].clone()
        out = torch.empty((m, 4), dtype=torch.float64, device=self.dev)
        for a in range(0, m, self.chunk):
            b = min(m, a + self.chunk)
            out[a:b] = self._run(x0[a:b], int(n_sectors))
        return out

    def _run(self, x0, ns):
        torch = _torch()
        from .constants import FFAG_ConversionTools
        from .coscan import crossing_states
        from .track import CrossingCapture, Pusher, _EphemeralBunch
        conv = FFAG_ConversionTools()
        m = x0.shape[0]
        P = x0[:, 4]
        v = P * conv.c ** 2 / torch.sqrt((P * conv.c) ** 2 + conv.E0 ** 2)
        mat = torch.zeros((m, 16), dtype=torch.float64, device=self.dev)
        mat[:, 0], mat[:, 1], mat[:, 2], mat[:, 3] = x0[:, 0], x0[:, 1] * v, x0[:, 2], x0[:, 3] * v
        mat[:, 5] = torch.sqrt(1.0 - x0[:, 1] ** 2 - x0[:, 3] ** 2) * v / x0[:, 0]
        mat[:, 7] = 1.0
        mat[:, 8] = 1.0
        T = ns * self.period
        w_min = float(mat[:, 5].min().item())
        nsteps = int(math.ceil(1.25 * T / (w_min * self.dt))) + 4
        b = _EphemeralBunch(mat, "Boris", self.dev)
        pu = Pusher(b, self.gp, "Boris", self.precision)
        cap = CrossingCapture(b, [T % (2 * np.pi)], self.gp, self.dt)
        xing = cap.prepare(nsteps)
        pu.push(self._clock_for(nsteps), 0, nsteps, 0, xing=xing)
        self.launches += 1
        k = int(cap.count.item())
        if k > cap.x.capacity:
            raise RuntimeError(f"crossing records overflowed: {k} > {cap.x.capacity}")
        rec = cap.buf[:k * _lib.CROSSING_RECORD].view(k, _lib.CROSSING_RECORD)
        rec = rec[(rec[:, 8] < T) & (rec[:, 15] >= T)]        # the step that passes T (unwrapped azimuth)
        idx = rec[:, 1].long()
        if idx.numel() != m or torch.unique(idx).numel() != m:
            raise RuntimeError(f"{m - torch.unique(idx).numel()} of {m} states did not reach the sector entrance")
        st = crossing_states(rec, self.dt, target=T)
        out = torch.empty((m, 4), dtype=torch.float64, device=self.dev)
        out[idx, 0] = st[:, 0]
        out[idx, 1] = st[:, 1] / v[idx]
        out[idx, 2] = st[:, 2]
        out[idx, 3] = st[:, 3] / v[idx]
        return out


# ------------------------------------------------------------- the frame
class SectorFrame:
    """Normalised coordinates at the sector entrance.

    u = r - r_co(e), pu = pr - pr_co(e) (closed orbit of the energy, a
    Chebyshev fit over the energy range), then Floquet coordinates of the
    mid-energy Twiss parameters, scaled so that amplitude 1 is the largest
    ellipse with |u| <= A_x and |pu| <= A_p (same for z, pz)."""

    def __init__(self, Ek_range, co_cheb_r, co_cheb_pr, twiss_x, twiss_z, amp, nsectors, tunes=None):
        self.Ek_range = (float(Ek_range[0]), float(Ek_range[1]))
        self.Emid = 0.5 * (self.Ek_range[0] + self.Ek_range[1])
        self.Ehalf = 0.5 * (self.Ek_range[1] - self.Ek_range[0])
        self.cr = np.asarray(co_cheb_r, np.float64)
        self.cpr = np.asarray(co_cheb_pr, np.float64)
        self.twiss = {"x": tuple(map(float, twiss_x)), "z": tuple(map(float, twiss_z))}
        self.amp = (float(amp[0]), float(amp[1]))
        self.nsectors = int(nsectors)
        self.tunes = tunes
        self.R = {}
        for pl, (al, be) in self.twiss.items():
            ga = (1 + al * al) / be
            self.R[pl] = min(self.amp[0] / math.sqrt(be), self.amp[1] / math.sqrt(ga))
        self.conv = FFAG_ConversionTools()

    # energies
    def e_of(self, Ek):
        return (Ek - self.Emid) / self.Ehalf

    def Ek_of(self, e):
        return self.Emid + self.Ehalf * e

    def P_of_Ek(self, Ek):
        return self.conv.Ek2P(Ek)

    def Ek_of_P(self, P):
        E0 = self.conv.E0
        return (np.sqrt((P * self.conv.c) ** 2 + E0 * E0) - E0) / 1e6 / self.conv.q if not hasattr(P, "sqrt") \
            else ((P * self.conv.c) ** 2 + E0 * E0).sqrt().sub(E0) / 1e6 / self.conv.q

    def co(self, e):
        """Closed orbit (r_co, pr_co) at energy coordinate e (numpy or torch)."""
        def cheb(c, x):
            b1 = b2 = 0.0 * x
            for ck in c[:0:-1]:
                b1, b2 = 2 * x * b1 - b2 + ck, b1
            return x * b1 - b2 + c[0]
        return cheb(self.cr, e), cheb(self.cpr, e)

    def to_norm(self, phys):
        """phys (n, 5) r, pr, z, pz, P (torch float64) -> s (n, 5)."""
        torch = _torch()
        e = self.e_of(self.Ek_of_P(phys[:, 4]))
        rco, prco = self.co(e)
        out = torch.empty_like(phys)
        for j, pl, a, b in ((0, "x", phys[:, 0] - rco, phys[:, 1] - prco), (2, "z", phys[:, 2], phys[:, 3])):
            al, be = self.twiss[pl]
            sb = math.sqrt(be)
            out[:, j] = a / sb / self.R[pl]
            out[:, j + 1] = (al * a + be * b) / sb / self.R[pl]
        out[:, 4] = e
        return out

    def to_phys(self, s, e):
        """s (n, >=4) normalised (any float type), e (n,) float64 -> (n, 4)
        r, pr, z, pz float64."""
        torch = _torch()
        s = s[:, :4].to(torch.float64)
        rco, prco = self.co(e)
        out = torch.empty((s.shape[0], 4), dtype=torch.float64, device=s.device)
        for j, pl in ((0, "x"), (2, "z")):
            al, be = self.twiss[pl]
            sb = math.sqrt(be)
            X, PX = s[:, j] * self.R[pl], s[:, j + 1] * self.R[pl]
            u = X * sb
            out[:, j] = u
            out[:, j + 1] = (PX * sb - al * u) / be
        out[:, 0] += rco
        out[:, 1] += prco
        return out

    def error(self, phys_a, phys_b, e):
        """Per-state error max(|dr|/r_co, |dpr|, |dz|/r_co, |dpz|)."""
        rco, _ = self.co(e)
        d = (phys_a - phys_b).abs()
        return _torch().stack([d[:, 0] / rco, d[:, 1], d[:, 2] / rco, d[:, 3]], 1).amax(1)

    @classmethod
    def build(cls, tracker, Ek_range=(300.0, 600.0), amp=(10e-3, 5e-3), r_guess=None, pr_guess=0.0,
              n_energies=17, degree=12):
        """Closed orbits (Newton on the S-step sector map) at Chebyshev nodes of
        the energy range, and the mid-energy Twiss parameters from the
        one-sector transfer matrix."""
        torch = _torch()
        conv = FFAG_ConversionTools()
        Emid, Ehalf = 0.5 * (Ek_range[0] + Ek_range[1]), 0.5 * (Ek_range[1] - Ek_range[0])
        nodes = np.cos(np.pi * (np.arange(n_energies) + 0.5) / n_energies)[::-1]
        Ek = Emid + Ehalf * nodes
        P = conv.Ek2P(Ek)
        r, pr = _closed_orbits(tracker, P, r_guess, pr_guess)
        cr = np.polynomial.chebyshev.chebfit(nodes, r, degree)
        cpr = np.polynomial.chebyshev.chebfit(nodes, pr, degree)
        # Twiss at mid energy from central differences
        Pm = float(conv.Ek2P(Emid))
        rm = float(np.polynomial.chebyshev.chebval(0.0, cr))
        prm = float(np.polynomial.chebyshev.chebval(0.0, cpr))
        dx = np.array([1e-6, 1e-7, 1e-6, 1e-7])
        x0 = np.tile([rm, prm, 0.0, 0.0, Pm], (8, 1))
        for j in range(4):
            x0[2 * j, j] += dx[j]
            x0[2 * j + 1, j] -= dx[j]
        x1 = tracker.run(torch.from_numpy(x0).to(tracker.dev), 1).cpu().numpy()
        M = np.zeros((4, 4))
        for j in range(4):
            M[:, j] = (x1[2 * j] - x1[2 * j + 1]) / (2 * dx[j])
        tw, tunes = [], []
        for blk in (M[:2, :2], M[2:, 2:]):
            c = 0.5 * np.trace(blk)
            if abs(c) >= 1:
                raise RuntimeError(f"unstable one-sector motion (|trace/2| = {abs(c):.4f})")
            sn = math.copysign(math.sqrt(1 - c * c), blk[0, 1])
            tw.append(((blk[0, 0] - blk[1, 1]) / (2 * sn), blk[0, 1] / sn))
            mu = math.atan2(sn, c) % (2 * np.pi)
            tunes.append(mu * tracker.nsectors / (2 * np.pi))
        return cls(Ek_range, cr, cpr, tw[0], tw[1], amp, tracker.nsectors, tunes=tunes)


def _closed_orbits(tracker, P, r_guess, pr_guess, iters=40, tol=1e-13):
    """Newton iteration of (r, pr) -> one-sector map at z = 0 for each
    momentum, finite-difference Jacobian, all momenta in one launch per pass;
    continuation from the lowest energy when no guess per momentum is given."""
    torch = _torch()
    P = np.asarray(P, np.float64)
    m = len(P)
    if r_guess is None:
        raise ValueError("a closed-orbit radius guess is required")
    r = np.broadcast_to(np.asarray(r_guess, np.float64), (m,)).copy()
    pr = np.broadcast_to(np.asarray(pr_guess, np.float64), (m,)).copy()
    dr, dp = 1e-6, 1e-7
    for _ in range(iters):
        x0 = np.zeros((3 * m, 5))
        x0[:, 4] = np.repeat(P, 3)
        x0[0::3, 0], x0[0::3, 1] = r, pr
        x0[1::3, 0], x0[1::3, 1] = r + dr, pr
        x0[2::3, 0], x0[2::3, 1] = r, pr + dp
        x1 = tracker.run(torch.from_numpy(x0).to(tracker.dev), 1).cpu().numpy()
        F = x1[0::3, :2] - x0[0::3, :2]
        a = (x1[1::3, :2] - x1[0::3, :2]) / dr
        b = (x1[2::3, :2] - x1[0::3, :2]) / dp
        a11, a21, a12, a22 = a[:, 0] - 1, a[:, 1], b[:, 0], b[:, 1] - 1
        det = a11 * a22 - a12 * a21
        d_r = -(a22 * F[:, 0] - a12 * F[:, 1]) / det
        d_p = -(-a21 * F[:, 0] + a11 * F[:, 1]) / det
        r, pr = r + d_r, pr + d_p
        if np.all(np.abs(F) < tol * np.maximum(1.0, np.abs(x0[0::3, :2]))):
            break
    if not np.all(np.isfinite(r)):
        raise RuntimeError("closed-orbit Newton iteration diverged")
    return r, pr


# ------------------------------------------------------------- data
def sample_domain(n, rng, radius=1.0):
    """Uniform in the normalised phase space: each transverse plane uniform
    in the disc of `radius`, e uniform in [-1, 1]."""
    s = np.zeros((n, 5))
    for j in (0, 2):
        rho = radius * np.sqrt(rng.random(n))
        ph = 2 * np.pi * rng.random(n)
        s[:, j], s[:, j + 1] = rho * np.cos(ph), rho * np.sin(ph)
    s[:, 4] = rng.uniform(-1.0, 1.0, n)
    return s


def make_dataset(frame, tracker, n, seed=0, radius=1.05, chunk=1 << 21):
    """n sector crossings: inputs X and targets T (float32 (n, 8) device
    tensors: s, then zero padding) from one sector of the plain tracker."""
    torch = _torch()
    rng = np.random.Generator(np.random.PCG64(seed))
    dev = tracker.dev
    X = torch.zeros((n, 8), dtype=torch.float32, device=dev)
    T = torch.zeros((n, 8), dtype=torch.float32, device=dev)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        s = torch.from_numpy(sample_domain(b - a, rng, radius)).to(dev)
        e = s[:, 4]
        phys = torch.empty((b - a, 5), dtype=torch.float64, device=dev)
        phys[:, :4] = frame.to_phys(s, e)
        phys[:, 4] = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(e.cpu().numpy())), device=dev)
        out = torch.empty_like(phys)
        out[:, :4] = tracker.run(phys, 1)
        out[:, 4] = phys[:, 4]
        s1 = frame.to_norm(out)
        X[a:b, :5] = s.float()
        T[a:b, :5] = s1.float()
    return X, T


# ------------------------------------------------------------- training
def skip_features(x):
    """[s0..s4, 1, s_i s_j (QUAD order)] of inputs x (n, >=5), float64."""
    torch = _torch()
    x = x[:, :5].double()
    return torch.cat([x, torch.ones_like(x[:, :1])] + [(x[:, i] * x[:, j])[:, None] for i, j in QUAD], 1)


def fit_skip(params, X, T, n_fit=4, max_rows=1 << 22, order=2):
    """Least-squares skip connection (float64 normal equations over up to
    max_rows samples): T[:, :n_fit] - X[:, :n_fit] ~ X Ws + bs (+ q(X) Wq
    for order 2)."""
    torch = _torch()
    A = skip_features(X[:max_rows])
    if order < 2:
        A = A[:, :6]
    Bm = (T[:max_rows, :n_fit] - X[:max_rows, :n_fit]).double()
    sol = torch.linalg.solve(A.T @ A, A.T @ Bm)
    for k in SKIP:
        block(params, k).zero_()
    block(params, "Ws")[:5, :n_fit] = sol[:5].float()
    block(params, "bs")[:n_fit] = sol[5].float()
    if order >= 2:
        block(params, "Wq")[:15, :n_fit] = sol[6:].float()


class Trainer:
    """Adam on the tensor-core forward/backward (ffa_mlp_train_step).

    lr_table (device float32, one learning rate per step) switches to the
    device schedule: step k takes lr_table[k] and Adam's bias corrections of
    step k + 1 from a device counter, so that graph_step can replay one
    captured CUDA graph of the whole step (about 30 launches) with nothing
    read from the host; step() then ignores its lr argument."""

    def __init__(self, params, batch=8192, n_fit=4, freeze_skip=True, beta1=0.9, beta2=0.999, eps=1e-8,
                 lr_table=None):
        torch = _torch()
        self.p = params
        dev = params.device
        self.lr_table = None if lr_table is None else lr_table.to(device=dev, dtype=torch.float32).contiguous()
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev) if lr_table is not None else None
        self._graph = None
        self.B, self.n_fit = int(batch), int(n_fit)
        self.g = torch.zeros_like(params)
        self.m = torch.zeros_like(params)
        self.v = torch.zeros_like(params)
        self.mask = torch.ones(N_PARAMS, dtype=torch.uint8, device=dev)
        if freeze_skip:
            for k in SKIP:
                block(self.mask, k).zero_()
        self.work = torch.empty(8 * self.B * HIDDEN + 24 * self.B + _lib.MLP_SPLIT_WORK, dtype=torch.float32,
                                device=dev)
        self.loss_part = torch.zeros(LOSS_PARTS, dtype=torch.float64, device=dev)
        self.beta1, self.beta2, self.eps = beta1, beta2, eps
        self.t = 0
        self.launches = 0

    def step(self, x, t, lr):
        """One step on the batch x, t ((B, 8) float32, contiguous); lr = 0
        computes loss and gradients only (host schedule)."""
        torch = _torch()
        assert x.shape[0] == self.B and x.is_contiguous() and t.is_contiguous()
        if lr > 0 or self.lr_table is not None:
            self.t += 1
        d = _lib.MlpTrainDesc()
        d.batch, d.n_fit, d.step = self.B, self.n_fit, max(self.t, 1)
        d.lr, d.beta1, d.beta2, d.eps = float(lr), self.beta1, self.beta2, self.eps
        d.params, d.grads, d.adam_m, d.adam_v = (self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
                                                 self.v.data_ptr())
        d.mask = self.mask.data_ptr()
        d.x, d.target = x.data_ptr(), t.data_ptr()
        d.work, d.loss_part = self.work.data_ptr(), self.loss_part.data_ptr()
        if self.lr_table is not None:
            d.lr_table, d.counter = self.lr_table.data_ptr(), self.counter.data_ptr()
        stream = torch.cuda.current_stream(self.p.device).cuda_stream
        _lib.check(_lib.lib().ffa_mlp_train_step(ctypes.byref(d), stream), "ffa_mlp_train_step")
        self.launches += 1

    def graph_step(self, x, t):
        """step() under the device schedule through a CUDA graph: the batch
        is copied into fixed buffers and the graph of one step replayed.  The
        first call runs the step directly (it also sets the kernels up) and
        captures the next one."""
        torch = _torch()
        if self.lr_table is None:
            raise ValueError("graph_step needs the device schedule (lr_table)")
        if self._graph is None:
            self._xb, self._tb = x.clone(), t.clone()
            self.step(self._xb, self._tb, 0.0)
            torch.cuda.current_stream(self.p.device).synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.step(self._xb, self._tb, 0.0)
            self.t -= 1                       # capturing ran nothing
            self.launches -= 1
            self._graph = g
            return
        self._xb.copy_(x)
        self._tb.copy_(t)
        self._graph.replay()
        self.t += 1
        self.launches += 1

    def mse(self):
        """Mean squared error of the last step's batch (before its update)."""
        return float(self.loss_part.sum().item()) / (self.B * self.n_fit)


def skip_map(params, X, n_fit=4):
    """The skip connection's output s + s Ws + bs + q(s) Wq (float64, first
    n_fit columns) for inputs X."""
    torch = _torch()
    W = torch.cat([block(params, "Ws")[:5, :n_fit], block(params, "bs")[None, :n_fit],
                   block(params, "Wq")[:15, :n_fit]], 0).double()
    return X[:, :n_fit].double() + skip_features(X) @ W


def residual_scale(params, X, T, n_fit=4, chunk=1 << 21):
    """Power of two nearest the rms of what the skip connection misses."""
    acc, cnt = 0.0, 0
    for a in range(0, X.shape[0], chunk):
        r = T[a:a + chunk, :n_fit].double() - skip_map(params, X[a:a + chunk], n_fit)
        acc += float((r * r).sum())
        cnt += r.numel()
    rms = math.sqrt(acc / max(cnt, 1))
    return 2.0 ** round(math.log2(rms)) if rms > 0 else 1.0


def lr_schedule(total, lr, lr_min, warmup):
    """Learning rate of steps 0..total-1: cosine from lr to lr_min over the
    run, times (k + 1) / warmup for the first `warmup` steps (float64)."""
    kk = np.arange(int(total))
    sched = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * kk / max(int(total), 1)))
    return np.where(kk < warmup, sched * (kk + 1) / warmup, sched)


def train(params, X, T, epochs=10, batch=8192, lr=2e-3, lr_min=1e-5, warmup=200, seed=0, n_fit=4,
          log_every=0, time_limit=None, eps=1e-8, out_scale="auto", chunk=1 << 21, graph=True):
    """Second-order skip connection by least squares, then Adam on the MLP
    with a cosine learning rate.

    The network is trained on what the skip connection misses divided by
    `out_scale` (by default the power of two nearest its rms), so that its
    output is of order one and the optimiser's step noise on W4 and b4 is
    not of the residual's own size; the scale is folded into W4 and b4 at the
    end (exactly: a power of two).  graph: the learning-rate schedule as a
    device table and every step after the first a replay of one captured
    CUDA graph (Trainer.graph_step); else one host-scheduled call per step.
    Returns the history [(step, mse)] of the scaled problem (sampled when
    log_every > 0) and the trainer."""
    torch = _torch()
    fit_skip(params, X, T, n_fit)
    sigma = residual_scale(params, X, T, n_fit, chunk) if out_scale == "auto" else float(out_scale or 1.0)
    if sigma != 1.0:
        Tn = T.clone()
        for a in range(0, X.shape[0], chunk):
            sk = skip_map(params, X[a:a + chunk], n_fit)
            Tn[a:a + chunk, :n_fit] = (sk + (T[a:a + chunk, :n_fit].double() - sk) / sigma).float()
        T = Tn
    n = X.shape[0]
    nb = n // batch
    total = max(1, epochs * nb)
    sched = lr_schedule(total, lr, lr_min, warmup)
    tr = Trainer(params, batch=batch, n_fit=n_fit, eps=eps,
                 lr_table=torch.from_numpy(sched.astype(np.float32)) if graph else None)
    tr.out_scale = sigma
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    hist = []
    t0 = time.perf_counter()
    k = 0
    done = False
    for ep in range(epochs):
        perm = torch.randperm(n, device=X.device, generator=g)
        Xs, Ts = X[perm].contiguous(), T[perm].contiguous()
        for i in range(nb):
            if graph:
                tr.graph_step(Xs[i * batch:(i + 1) * batch], Ts[i * batch:(i + 1) * batch])
            else:
                tr.step(Xs[i * batch:(i + 1) * batch], Ts[i * batch:(i + 1) * batch], float(sched[k]))
            k += 1
            if log_every and k % log_every == 0:
                hist.append((k, tr.mse()))
            if time_limit is not None and k % 64 == 0 and time.perf_counter() - t0 > time_limit:
                done = True
                break
        if done:
            break
    if sigma != 1.0:
        block(params, "W4").mul_(sigma)
        block(params, "b4").mul_(sigma)
    return hist, tr


def evaluate(params, X, T, n_fit=4, batch=8192):
    """Mean squared error of the network over (X, T) (lr = 0 steps)."""
    tr = Trainer(params, batch=batch, n_fit=n_fit)
    nb = X.shape[0] // batch
    tot = 0.0
    for i in range(nb):
        tr.step(X[i * batch:(i + 1) * batch].contiguous(), T[i * batch:(i + 1) * batch].contiguous(), 0.0)
        tot += tr.mse()
    return tot / max(nb, 1)


# ------------------------------------------------------------- inference
class LearnedSectorMap:
    """Tracking with the learned map, audited against the plain tracker."""

    def __init__(self, frame, tracker, params, radius=1.0, audit_every=50, audit_frac=0.01, audit_tol=1e-5,
                 seed=0):
        torch = _torch()
        self.frame, self.tracker = frame, tracker
        self.p = params
        self.dev = params.device
        self.radius2 = float(radius) ** 2
        self.audit_every, self.audit_frac, self.audit_tol = int(audit_every), float(audit_frac), float(audit_tol)
        self.wpack = torch.empty(_lib.MLP_WPACK_BYTES, dtype=torch.uint8, device=self.dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.rng = np.random.Generator(np.random.PCG64(seed))
        self.launches = 0
        self.pack()

    def pack(self):
        torch = _torch()
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        _lib.check(_lib.lib().ffa_mlp_pack(self.p.data_ptr(), self.wpack.data_ptr(), stream), "ffa_mlp_pack")
        self.launches += 1

    def apply(self, state, n_apply, applied=None, radius2=None):
        """n_apply maps in place on state ((n, 8) float32 device)."""
        torch = _torch()
        assert state.dtype == torch.float32 and state.is_contiguous() and state.shape[1] == 8
        d = _lib.MlpInferDesc()
        d.n, d.n_apply = state.shape[0], int(n_apply)
        d.radius2 = self.radius2 if radius2 is None else float(radius2)
        d.params, d.wpack, d.state = self.p.data_ptr(), self.wpack.data_ptr(), state.data_ptr()
        d.applied = applied.data_ptr() if applied is not None else None
        d.error = self.err.data_ptr()
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        _lib.check(_lib.lib().ffa_mlp_infer(ctypes.byref(d), stream), "ffa_mlp_infer")
        self.launches += 1

    def error_flag(self):
        """Non-zero when an inference launch gave up on a pipeline wait."""
        return int(self.err.item())

    def track(self, phys, turns, record=False):
        """phys (n, 5) r, pr, z, pz, P at a sector entrance (float64).  Returns
        a dict: 'phys' (n, 4) after `turns` turns, 'plain' (n,) bool (states
        the plain tracker finished), 'audits' [(turn, sampled, failed,
        max_error)], 'record' (turns + 1, n, 4) normalised transverse
        coordinates after every turn when record=True."""
        torch = _torch()
        dev = self.dev
        phys = torch.as_tensor(phys, dtype=torch.float64, device=dev)
        n = phys.shape[0]
        N = self.frame.nsectors
        s = self.frame.to_norm(phys)
        e = s[:, 4].clone()
        P = phys[:, 4].clone()
        state = torch.zeros((n, 8), dtype=torch.float32, device=dev)
        state[:, :5] = s.float()
        plain = torch.zeros(n, dtype=torch.bool, device=dev)
        plain_phys = torch.zeros((n, 4), dtype=torch.float64, device=dev)
        applied = torch.empty(n, dtype=torch.int32, device=dev)
        audits = []
        rec = [self._norm4(state, plain, plain_phys, e, P).cpu()] if record else None
        step_turns = 1 if record else self.audit_every
        turn = 0
        while turn < turns:
            nt = min(step_turns, turns - turn, self.audit_every - turn % self.audit_every)
            napp = nt * N
            self.apply(state, napp, applied)
            # states that left the domain: the plain tracker finishes their sectors
            need = ((applied < napp) & ~plain).nonzero().flatten()
            if need.numel():
                rem = napp - applied[need].long()
                ph = self.frame.to_phys(state[need], e[need])
                for r_ in torch.unique(rem).tolist():
                    sel = (rem == r_).nonzero().flatten()
                    x0 = torch.cat([ph[sel], P[need][sel, None]], 1)
                    ph[sel] = self.tracker.run(x0, int(r_))
                plain_phys[need] = ph
                plain[need] = True
                state[need, 4] = float("inf")      # outside the domain from now on
            old = (plain & (applied == 0)).nonzero().flatten()
            old = old[~torch.isin(old, need)] if need.numel() else old
            if old.numel():
                plain_phys[old] = self.tracker.run(torch.cat([plain_phys[old], P[old, None]], 1), napp)
            turn += nt
            if turn % self.audit_every == 0:
                audits.append(self._audit(turn, state, plain, plain_phys, e, P))
            if record:
                rec.append(self._norm4(state, plain, plain_phys, e, P).cpu())
        if self.error_flag():
            raise _lib.FFAError("ffa_mlp_infer: a pipeline wait timed out")
        out = self.frame.to_phys(state, e)
        out[plain] = plain_phys[plain]
        res = {"phys": out, "plain": plain, "audits": audits}
        if record:
            res["record"] = torch.stack(rec).numpy()
        return res

    def _norm4(self, state, plain, plain_phys, e, P):
        s = state[:, :4].double().clone()
        if plain.any():
            idx = plain.nonzero().flatten()
            s[idx] = self.frame.to_norm(_torch().cat([plain_phys[idx], P[idx, None]], 1))[:, :4]
        return s.float()

    def _audit(self, turn, state, plain, plain_phys, e, P):
        torch = _torch()
        live = (~plain).nonzero().flatten()
        if live.numel() == 0:
            return (turn, 0, 0, 0.0)
        k = max(1, int(round(self.audit_frac * live.numel())))
        pick = live[torch.as_tensor(self.rng.choice(live.numel(), size=k, replace=False), device=self.dev)]
        st = state[pick].clone()
        app = torch.empty(k, dtype=torch.int32, device=self.dev)
        self.apply(st, 1, app)
        ph0 = self.frame.to_phys(state[pick], e[pick])
        ref = self.tracker.run(torch.cat([ph0, P[pick, None]], 1), 1)
        got = self.frame.to_phys(st, e[pick])
        err = self.frame.error(got, ref, e[pick])
        err = torch.where(app == 1, err, torch.full_like(err, float("inf")))
        bad = pick[err > self.audit_tol]
        if bad.numel():
            plain_phys[bad] = self.frame.to_phys(state[bad], e[bad])
            plain[bad] = True
            state[bad, 4] = float("inf")
        return (turn, k, int(bad.numel()), float(err[torch.isfinite(err)].max().item()) if torch.isfinite(err).any()
                else float("inf"))


def plain_track(frame, tracker, phys, turns, record=False):
    """The FP64 reference: every state through `turns` turns of the plain
    tracker (one launch per turn); same outputs as LearnedSectorMap.track."""
    torch = _torch()
    phys = torch.as_tensor(phys, dtype=torch.float64, device=tracker.dev)
    x = phys.clone()
    rec = [frame.to_norm(x)[:, :4].float().cpu()] if record else None
    for _ in range(turns):
        x[:, :4] = tracker.run(x, frame.nsectors)
        if record:
            rec.append(frame.to_norm(x)[:, :4].float().cpu())
    res = {"phys": x[:, :4].clone()}
    if record:
        res["record"] = torch.stack(rec).numpy()
    return res


# ------------------------------------------- the time-domain plain pushers
def phys_to_boris(phys, conv=None) -> np.ndarray:
    """States at a sector entrance, phys (n, 5) r, pr, z, pz, P (pr, pz the
    transverse momenta over P, P in kg m/s), as the Boris pushers' N x 16
    matrix at fi = 0: vr = pr v, vz = pz v, dfi/dt = sqrt(1 - pr^2 - pz^2) v / r,
    all injected and alive."""
    from .constants import FFAG_ConversionTools
    conv = conv or FFAG_ConversionTools()
    ph = np.asarray(phys.cpu().numpy() if hasattr(phys, "cpu") else phys, np.float64)
    E = np.sqrt((ph[:, 4] * conv.c) ** 2 + conv.E0 ** 2)
    v = ph[:, 4] * conv.c ** 2 / E
    m = np.zeros((ph.shape[0], 16))
    m[:, 0] = ph[:, 0]
    m[:, 1] = ph[:, 1] * v
    m[:, 2] = ph[:, 2]
    m[:, 3] = ph[:, 3] * v
    m[:, 5] = np.sqrt(1.0 - ph[:, 1] ** 2 - ph[:, 3] ** 2) * v / ph[:, 0]
    m[:, 7] = 1.0
    m[:, 8] = 1.0
    m[:, 15] = np.arange(ph.shape[0])
    return m


def boris_record(frame, gp, phys, turns, dt, precision="fp64", device=None):
    """The time-domain Boris pusher on the states `phys` (sector entrance,
    fi = 0) for enough steps that every state makes `turns` turns; the
    normalised transverse coordinates where each state crosses fi = 0,
    turn by turn (turns + 1, n, 4) as LearnedSectorMap.track records them
    (NaN for a state lost before)."""
    import os
    import tempfile
    torch = _torch()
    from . import diagnostics
    from .bunch import FFAG_Bunch
    from .dump import Dumps, PositionDumpBunch
    from .track import FFAG_RungeKutta
    m = phys_to_boris(phys)
    n = m.shape[0]
    t_rev = (2 * np.pi / m[:, 5]).max()            # the slowest state's revolution time, roughly
    nsteps = int(np.ceil((turns + 0.5) * t_rev / dt))
    b = FFAG_Bunch(m, BunchType="Boris", device=device)
    d = PositionDumpBunch(0.0, -dt, (nsteps + 1) * dt, save_folder=os.path.join(tempfile.mkdtemp(), "x"))
    dumps = Dumps()
    dumps.add_dump(d)
    lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
          "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": dumps}
    FFAG_RungeKutta(precision=precision, verbose=False).rk4_solve_dt_bunch3_withSC_boris(None, 0.0, b, gp, lp)
    tab = diagnostics.crossing_table(d.crossing_records, n, dt)[: turns + 1]
    rec = np.full((turns + 1, n, 4), np.nan, np.float32)
    P = np.asarray(phys[:, 4].cpu().numpy() if hasattr(phys, "cpu") else phys[:, 4], np.float64)
    for t in range(tab.shape[0]):
        ok = np.isfinite(tab[t, :, 0])
        if not ok.any():
            continue
        spd = tab[t, ok, 4]
        ph = np.stack([tab[t, ok, 0], tab[t, ok, 1] / spd, tab[t, ok, 2], tab[t, ok, 3] / spd, P[ok]], 1)
        rec[t, ok] = frame.to_norm(torch.as_tensor(ph, dtype=torch.float64))[:, :4].float().numpy()
    return rec


# ------------------------------------------------------------- persistence
def save(path, params, frame):
    """Writes a trained network and its coordinate frame to one .npz file."""
    p = params.detach().cpu().numpy() if hasattr(params, "detach") else np.asarray(params, np.float32)
    np.savez(path, params=p.astype(np.float32), Ek_range=np.array(frame.Ek_range), cheb_r=frame.cr,
             cheb_pr=frame.cpr, twiss_x=np.array(frame.twiss["x"]), twiss_z=np.array(frame.twiss["z"]),
             amp=np.array(frame.amp), nsectors=np.array(frame.nsectors),
             tunes=np.array(frame.tunes if frame.tunes is not None else [np.nan, np.nan]))


def load(path):
    """(params float32 numpy (N_PARAMS,), SectorFrame) from a file of save()."""
    d = np.load(path)
    if d["params"].shape != (N_PARAMS,):
        raise ValueError(f"{path}: {d['params'].shape[0]} parameters, this library uses {N_PARAMS}")
    frame = SectorFrame(tuple(d["Ek_range"]), d["cheb_r"], d["cheb_pr"], tuple(d["twiss_x"]), tuple(d["twiss_z"]),
                        tuple(d["amp"]), int(d["nsectors"]), tunes=list(d["tunes"]))
    return d["params"].copy(), frame


# ------------------------------------------------------------- diagnostics
def tunes(record, nsectors=None):
    """Fractional tunes per state from turn-by-turn Floquet coordinates
    record (T + 1, n, 4): mean per-turn phase advance of X - i PX (and of
    the vertical pair), in [0, 1)."""
    rec = np.asarray(record, np.float64)
    out = []
    for j in (0, 2):
        z = rec[:, :, j] - 1j * rec[:, :, j + 1]
        dphi = np.angle(z[1:] / z[:-1]) % (2 * np.pi)
        out.append(dphi.mean(0) / (2 * np.pi))
    return np.stack(out, 1)


def betatron_emittance(frame, s4):
    """rms emittances of the betatron motion from normalised transverse
    coordinates s4 (n, 4) (closed orbit of each energy removed, mid-energy
    Twiss frame): R^2 times the rms emittance of (X, PX) and (Y, PY)."""
    s4 = np.asarray(s4, np.float64)
    return rms_emittance(s4) * np.array([frame.R["x"] ** 2, frame.R["z"] ** 2])


def rms_emittance(phys):
    """rms emittances (x: r, pr; z: z, pz) of a set of states (n, >=4)."""
    a = np.asarray(phys, np.float64)
    out = []
    for j in (0, 2):
        u = a[:, j] - a[:, j].mean()
        p = a[:, j + 1] - a[:, j + 1].mean()
        out.append(math.sqrt(max(0.0, np.mean(u * u) * np.mean(p * p) - np.mean(u * p) ** 2)))
    return np.array(out)
