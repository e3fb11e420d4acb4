"""Particle container on the GPU.

FFAG_Bunch mirrors the reference's container (src/FFAG_Bunch.py:77-409): it
is built from the N x 16 v-format matrix, keeps the same injection and
survival bookkeeping, and exposes ``LocalBunch`` as the N x 16 float64 matrix
(assembled on demand).  The state itself lives in HBM as structure-of-arrays
float64 columns so that every kernel reads and writes coalesced words.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .constants import COLUMNS, NCOL, Q, C_LIGHT, E0_MEV


def injection_steps(inj_t_sorted: np.ndarray, t_lo: np.ndarray, t_hi: np.ndarray, step0: int, head: int) -> np.ndarray:
    """Step index at which each particle is injected, or -1.

    The reference injects, at the step whose start time is t, the particles
    from its injection head onwards with inj_t in [(t - dt) * 1e9, t * 1e9]
    (np.searchsorted left / right on the inj_t-sorted bunch) and moves the
    head past them (InjectParticles, src/FFAG_Bunch.py:265-303).  Because the
    windows advance monotonically, particle k is injected at the first step
    whose upper bound reaches inj_t[k], provided that step's lower bound does
    not exceed it; earlier particles skipped by a window are never injected.
    t_lo / t_hi are the window bounds in ns for steps step0, step0+1, ...
    """
    n = inj_t_sorted.shape[0]
    out = np.full(n, -1, dtype=np.int64)
    if n == 0 or len(t_hi) == 0:
        return out
    cand = np.searchsorted(t_hi, inj_t_sorted[head:], side="left")
    ok = cand < len(t_hi)
    lo_at = np.where(ok, t_lo[np.minimum(cand, len(t_hi) - 1)], np.inf)
    ok &= lo_at <= inj_t_sorted[head:]
    out[head:][ok] = cand[ok] + step0
    return out


class FFAG_Bunch:
    """Bunch of macroparticles; `ParticlesDistribution` is the v-format
    N x 16 matrix (Boris: col 5 = dfi/dt; RK4: col 5 = Etot [J]) sorted by
    inj_t.  `sc_grid_size` = (ns, nx, nz, sigma_ratio)."""

    def __init__(self, ParticlesDistribution, marcosize=1, sc_grid_size=(64, 128, 128, 12.0), BunchType="Boris",
                 device=None, rank=0, world_size=1):
        import torch
        a = np.ascontiguousarray(np.asarray(ParticlesDistribution, dtype=np.float64))
        if a.ndim != 2 or a.shape[1] < NCOL:
            raise ValueError("particle matrix must be N x 16")
        a = a[:, :NCOL]
        if BunchType not in ("Boris", "RK4"):
            raise ValueError("BunchType must be Boris or RK4")
        self.BunchType = BunchType
        self.TotalParticleNum = a.shape[0]
        # particles are split across ranks as FFAG_MPI.DivideVariables does
        # (src/FFAG_track.py:1126-1139): contiguous blocks, remainder round-robin
        gid = a[:, COLUMNS["Global_ID"]]
        local = divide_variables(len(gid), rank, world_size)
        a = a[local].copy()
        a[:, COLUMNS["Local_ID"]] = np.arange(a.shape[0])
        self.StaticBunchLocal = a.copy()
        self.TotalParticleNum_Local = a.shape[0]
        self.marcosize = marcosize
        self.speed_c = C_LIGHT
        self.q_charge = Q
        self.E0_rest_MeV = E0_MEV
        self.f_grid_size, self.x_grid_size, self.z_grid_size = int(sc_grid_size[0]), int(sc_grid_size[1]), int(sc_grid_size[2])
        self.sigma_ratio = float(sc_grid_size[3])
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._host_static = a  # cols 6, 13-15 never change on the device
        self._inj_t = np.ascontiguousarray(a[:, COLUMNS["inj_t"]])
        if np.any(np.diff(self._inj_t) < 0):
            raise ValueError("the bunch must be sorted by inj_t (column 6)")
        self._alloc(a)
        self._uninject_head = 0
        self.uninject_num = self.TotalParticleNum_Local
        self.InjectedNum_Local = 0
        self.SurvivedNum_Local = 0
        self.LostNum_Local = 0
        self.InjectedNum = self.SurvivedNum = self.LostNum = 0
        self.SEO_fi_axis = self.SEO_Ek_axis = self.SEO_r_matrix = self.SEO_pr_matrix = self.SEO_perimeter = None

    # ------------------------------------------------------------ storage
    def _alloc(self, a):
        import torch
        n = a.shape[0]
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.cols = {}
        for name, c in (("r", 0), ("vr", 1), ("z", 2), ("vz", 3), ("fi", 4), ("f5", 5), ("rf", 9),
                        ("esc_r", 10), ("esc_z", 11), ("esc_fi", 12)):
            self.cols[name] = torch.from_numpy(np.ascontiguousarray(a[:, c])).to(dev)
        self.cols["inj"] = torch.from_numpy((a[:, 7] == 1.0).astype(np.uint8)).to(dev)
        self.cols["surv"] = torch.from_numpy((a[:, 8] == 1.0).astype(np.uint8)).to(dev)
        self.cols["inj_step"] = torch.full((n,), -1, dtype=torch.int32, device=dev)
        for name in ("e_pre_r", "e_pre_z", "e_pre_fi", "e_pp_r", "e_pp_z", "e_pp_fi"):
            self.cols[name] = torch.zeros(n, **f64)
        self.cols["sc_pre"] = torch.zeros(n, dtype=torch.uint8, device=dev)
        self.cols["sc_pp"] = torch.zeros(n, dtype=torch.uint8, device=dev)
        self.status = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int64, device=dev)
        self._soa = None

    def soa(self) -> "_lib.StateSoA":
        if self._soa is None:
            s = _lib.StateSoA()
            for name, _ in _lib.StateSoA._fields_:
                t = self.cols.get(name)
                setattr(s, name, t.data_ptr() if t is not None else None)
            self._soa = s
        return self._soa

    @property
    def n(self) -> int:
        return self.TotalParticleNum_Local

    # --------------------------------------------------- injection schedule
    def set_injection_schedule(self, t_lo_ns: np.ndarray, t_hi_ns: np.ndarray, step0: int) -> None:
        """Uploads inj_step for the steps covered by the window bounds."""
        import torch
        steps = injection_steps(self._inj_t, t_lo_ns, t_hi_ns, step0, self._uninject_head)
        if steps.size and steps.max() > np.iinfo(np.int32).max:
            raise ValueError("step index exceeds int32")
        self.cols["inj_step"].copy_(torch.from_numpy(steps.astype(np.int32)))
        inj = steps >= 0
        if inj.any():
            self._uninject_head = int(np.nonzero(inj)[0].max()) + 1
        self._scheduled = steps

    def note_injected_until(self, step_end: int) -> None:
        """Host bookkeeping of particles injected at steps < step_end."""
        s = getattr(self, "_scheduled", None)
        if s is None:
            return
        done = (s >= 0) & (s < step_end)
        k = int(done.sum()) - getattr(self, "_counted", 0)
        if k > 0:
            self.InjectedNum_Local += k
            self.SurvivedNum_Local += k
            self.uninject_num -= k
            self._counted = getattr(self, "_counted", 0) + k

    def reset_schedule_count(self):
        self._counted = 0

    # ------------------------------------------------------------- views
    def alive_at_step(self, step: int) -> np.ndarray:
        """Survival flags at the start of absolute step `step` after that
        step's injection (the reference's Step_SurviveFlag), read before the
        step is pushed."""
        surv = self.cols["surv"].cpu().numpy().astype(bool)
        return surv | (self.cols["inj_step"].cpu().numpy() == step)

    @property
    def LocalBunch(self) -> np.ndarray:
        """The N x 16 v-format matrix (device -> host copy)."""
        import torch
        out = self._host_static.copy()
        for name, c in (("r", 0), ("vr", 1), ("z", 2), ("vz", 3), ("fi", 4), ("f5", 5), ("rf", 9),
                        ("esc_r", 10), ("esc_z", 11), ("esc_fi", 12)):
            out[:, c] = self.cols[name].cpu().numpy()
        out[:, 7] = self.cols["inj"].cpu().numpy().astype(np.float64)
        out[:, 8] = self.cols["surv"].cpu().numpy().astype(np.float64)
        return out

    def load_matrix(self, a: np.ndarray) -> None:
        """Replaces the device state with the N x 16 matrix `a`."""
        import torch
        a = np.asarray(a, dtype=np.float64)
        for name, c in (("r", 0), ("vr", 1), ("z", 2), ("vz", 3), ("fi", 4), ("f5", 5), ("rf", 9),
                        ("esc_r", 10), ("esc_z", 11), ("esc_fi", 12)):
            self.cols[name].copy_(torch.from_numpy(np.ascontiguousarray(a[:, c])))
        self.cols["inj"].copy_(torch.from_numpy((a[:, 7] == 1.0).astype(np.uint8)))
        self.cols["surv"].copy_(torch.from_numpy((a[:, 8] == 1.0).astype(np.uint8)))

    def restore_from_restart_matrix(self, *, assert_monotonic=True) -> None:
        """Recovers the injection head and counters from the flags of a
        restarted bunch (src/FFAG_Bunch.py:305-366)."""
        c = restart_counters(self._host_static, assert_monotonic=assert_monotonic)
        self._uninject_head = c["head"]
        self.InjectedNum_Local = c["injected"]
        self.uninject_num = c["uninjected"]
        self.SurvivedNum_Local = c["survived"]
        self.LostNum_Local = c["lost"]

    def status_counts(self) -> dict:
        s = self.status.cpu().numpy()
        return {"lost": int(s[_lib.STATUS_LOST]), "nan": int(s[_lib.STATUS_NAN]),
                "out_of_map": int(s[_lib.STATUS_OUT_OF_MAP]), "sc_degenerate": int(s[_lib.STATUS_SC_DEGENERATE])}

    def UpdateParticleNumGlobal(self, comm=None) -> None:
        """Survival counters from the device flags (src/FFAG_Bunch.py:369-392);
        with a torch.distributed group the counts are summed over ranks."""
        import torch
        inj = self.cols["inj"]
        surv = self.cols["surv"]
        injected = int((inj == 1).sum().item())
        survived = int(((inj == 1) & (surv == 1)).sum().item())
        self.InjectedNum_Local = injected
        self.SurvivedNum_Local = survived
        self.LostNum_Local = injected - survived
        vals = torch.tensor([injected, survived, injected - survived], dtype=torch.int64)
        if comm is not None:
            comm.all_reduce(vals)
        self.InjectedNum, self.SurvivedNum, self.LostNum = (int(v) for v in vals.tolist())


def restart_counters(a: np.ndarray, assert_monotonic: bool = True) -> dict:
    """Injection head and counters of an inj_t-sorted restart matrix: the
    head is the first particle not injected; the flags must form a step
    function [1 ... 1, 0 ... 0] along the matrix (src/FFAG_Bunch.py:305-366)."""
    N = a.shape[0]
    inj = a[:, COLUMNS["Inj_flag"]] > 0.5
    sur = a[:, COLUMNS["Survive"]] > 0.5
    zeros = np.flatnonzero(~inj)
    head = int(zeros[0]) if zeros.size else N
    if assert_monotonic:
        ok = (inj[:head].all() and (~inj[head:]).all()) if head < N else inj.all()
        if not ok:
            raise RuntimeError(
                "Restart bunch violates the designed structure: Inj_flag is not a step function "
                "along inj_t-sorted LocalBunch.")
    injected = int(inj.sum())
    return {"head": head, "injected": injected, "uninjected": int(N - injected), "survived": int(sur.sum()),
            "lost": int((inj & ~sur).sum())}


def divide_variables(total: int, rank: int, size: int) -> np.ndarray:
    """Indices owned by `rank` (FFAG_MPI.DivideVariables, src/FFAG_track.py:1126-1139)."""
    per = total // size
    mod = total - per * size
    idx = list(range(rank * per, (rank + 1) * per))
    if rank < mod:
        idx.append(per * size + rank)
    return np.array(idx, dtype=np.int64)
