#!/usr/bin/env python
"""Benchmark of the tracking hot path: particle-turns/s on one B200.

Workload (the multiparticle configuration the metric is quoted on):
12-sector scaling FFAG, proton 300 MeV, full 1301 x 6000 mid-plane map with
z-Taylor order 2 (z^4 in Bz, z^5 in Br/Bfi), two RF gaps at 100 kV
(reference semantics: the last gap's field wins), 1e5-particle seeded 6D
Gaussian on the closed orbit, 720 steps per turn, relativistic Boris in
float64.  One benchmark step = one turn = 720 fused push steps over the
whole bunch, inputs resident in HBM; L2 is flushed between timed steps.

`--impl reference` times the reference's algorithm on the host cores (the
C restatement in oracle/, all threads) on a bounded sample of the same
workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

N_PARTICLES = 100_000
STEPS_PER_TURN = 720
REF_SAMPLE_STEPS = 72       # steps of a turn the reference arm runs per step
MAX_ORDER = 2
# algorithmic float64 operations per particle-step of one Boris step: the
# arithmetic of the reference's step (field, RF kick, Cartesian round trip,
# Boris push; transcendentals not counted), the roofline's numerator
FP64_FLOP_PER_PARTICLE_STEP = 300.0
# the kernel's executed float64 operations per particle-step (2 per DFMA, 1
# per DADD / DMUL), counted by ncu on this workload: reported beside it
FP64_EXEC_FLOP_PER_PARTICLE_STEP = 419.4
# algorithmic float64 operations per particle-step of one RK4 step: four
# right-hand sides (azimuth mod sector 3, analytic field 93, z-Taylor sum 77,
# RF window test 4, equations of motion 40) and the stage arithmetic (k = h d,
# the stage states and the weighted sum, seven components each: 112), i.e.
# 4 x 217 + 112
RK4_FLOP_PER_PARTICLE_STEP = 980.0
# DRAM bytes (read + write) of one launch (one turn, 1e5 particles) from an
# ncu capture of the same launch, L2 flushed before it
BORIS_TRAFFIC_PER_LAUNCH = 19.571e6
# algorithmic HBM bytes per particle per launch: SoA state read
# (10 float64 + 2 flag bytes + int32 injection step) and written (10 float64 + 2 bytes)
STATE_BYTES_PER_PARTICLE = (10 * 8 + 2 + 4) + (10 * 8 + 2)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32c"])
    ap.add_argument("--n", type=int, default=N_PARTICLES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sc", action="store_true")
    ap.add_argument("--no-fp32c", action="store_true")
    ap.add_argument("--no-mapgen", action="store_true")
    ap.add_argument("--no-scan", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-coscan", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-rk4", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--learned-samples", type=int, default=20_000_000)
    ap.add_argument("--learned-epochs", type=int, default=8)
    ap.add_argument("--learned-n", type=int, default=10_000_000)
    return ap.parse_args()


def workload(seed=7, n=N_PARTICLES):
    import warnings
    warnings.simplefilter("ignore")
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools, FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical, FFAG_EField_new
    cfg = synthetic.lattice_bmap()
    bm = FFAG_Bfield_analytical(config=cfg, max_order=MAX_ORDER, stacks=synthetic.taylor_stacks(cfg, MAX_ORDER))
    em = FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=True)
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    gp.AddEMap(em)
    gp.AddAperture(7.5, 9.5, -0.1, 0.1)
    p = synthetic.centred_bunch(n, seed=seed)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    dt = synthetic.design_dt(300.0, STEPS_PER_TURN)
    return gp, v, dt


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return self
        # nvidia-smi takes a moment to start: wait (at most 5 s) for its
        # first sample so that the timed region is covered
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            self.fh.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_peak_tflops(dev_index):
    """FP64 FMA pipe peak measured live with the probe kernel."""
    import ctypes
    import torch
    from pyffa_b200 import build
    L = ctypes.CDLL(build.build_probe())
    L.ffa_probe_fp64_fma.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_float)]
    sms = torch.cuda.get_device_properties(dev_index).multi_processor_count
    blocks, iters = sms * 8, 4096
    out = torch.zeros(blocks, dtype=torch.float64, device="cuda")
    ms = ctypes.c_float()
    best = 0.0
    for _ in range(3):
        L.ffa_probe_fp64_fma(blocks, iters, ctypes.c_void_p(out.data_ptr()),
                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(ms))
        flops = 2.0 * 8 * iters * blocks * 256
        best = max(best, flops / (ms.value * 1e-3) / 1e12)
    return best


def fp32_peak_tflops(dev_index):
    """FP32 FMA pipe peak measured live with the probe kernel."""
    import ctypes
    import torch
    from pyffa_b200 import build
    L = ctypes.CDLL(build.build_probe())
    L.ffa_probe_fp32_fma.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_float)]
    sms = torch.cuda.get_device_properties(dev_index).multi_processor_count
    blocks, iters = sms * 8, 8192
    out = torch.zeros(blocks, dtype=torch.float32, device="cuda")
    ms = ctypes.c_float()
    best = 0.0
    for _ in range(3):
        L.ffa_probe_fp32_fma(blocks, iters, ctypes.c_void_p(out.data_ptr()),
                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(ms))
        flops = 2.0 * 8 * iters * blocks * 256
        best = max(best, flops / (ms.value * 1e-3) / 1e12)
    return best


def cpu_baseline(gp, v, dt, sample_n=100_000, steps=8 * STEPS_PER_TURN):
    """The reference algorithm on the host cores (oracle port, all threads):
    particle-turns/s on a bounded sample of the workload."""
    from oracle import oracle as O
    O.build()
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    m = np.ascontiguousarray(v[:sample_n].copy())
    O.boris_step(S, m[:64].copy(), 0.0, dt)  # warm the library
    t0 = time.perf_counter()
    O.track(S, "Boris", m, 0.0, dt, steps)
    el = time.perf_counter() - t0
    return {"value": sample_n * steps / STEPS_PER_TURN / el, "unit": "particle-turns/s", "cores": O.num_threads(),
            "kind": "port", "sample": f"{sample_n} particles x {steps} Boris steps ({steps // STEPS_PER_TURN} turns) of the "
                                "same workload",
            "seconds": el}


def sc_workload(n=1_000_000, seed=11):
    """c2: 1e6 macroparticles for 1e13 protons at 300 MeV, KV transverse with
    4 mm radii, Gaussian sigma_t = 20 ns, 64 slices on a 128 x 128 grid."""
    import warnings
    warnings.simplefilter("ignore")
    from pyffa_b200 import orbit, synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    t = orbit.seo_tables(synthetic.lattice_bmap(), np.linspace(280.0, 320.0, 9), nfi=721)
    seo = {k: t[k] for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}
    p = synthetic.centred_bunch(n, seed=seed, kind="kv", a_x=4e-3, a_z=4e-3, sig_t=20e-9, fi0=np.pi)
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    return v, seo


# Compulsory HBM bytes of one space-charge update of this design, per
# particle: pass 1 reads r, vr, z, vz, fi, f5 and the survival flag and writes
# x = r - r0 and pr0 (65 B); the deposit reads the flag, fi, x and z and
# writes the slice and cell indices (37 B); gather + roll read the slice, x,
# z, pr0, the flag, the pre mask and the three pre endpoints and write the
# three fields, both endpoint triples and both masks (128 B).  Per cell: the
# float32 charge, potential and field cubes, written once (16 B).  The
# fixed-point accumulator and the slices' spectra stay in L2 / shared memory.
SC_BYTES_PER_PARTICLE = 65 + 37 + 128
SC_BYTES_PER_CELL = 16
SC_GRID = (64, 128, 128)


def sc_bench(gp, dt, dev, hbm_peak, updates=20, warmup=3, turns=2):
    """c2 space charge: update time (ms) and HBM roofline of the periodic and
    the open-boundary solve on 1e6 macroparticles, 64 slices, 128 x 128;
    the c2 cycle (per turn 12 x (open-boundary update + 60 Boris steps, the
    field extrapolated between updates)) with the FP32C pusher, and with the
    FP64 pusher for comparison; and the fraction of the bunch that survives
    one cycle turn at the full charge, at 1e-3 of it, and without space
    charge (the aperture losses of the space-charge defocusing)."""
    import torch
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.space_charge import SpaceCharge
    from pyffa_b200.track import Pusher, StepClock
    v, seo = sc_workload()
    n = v.shape[0]
    cells = SC_GRID[0] * SC_GRID[1] * SC_GRID[2]
    nbytes = SC_BYTES_PER_PARTICLE * n + SC_BYTES_PER_CELL * cells
    out = {"particles": n, "grid": list(SC_GRID), "sigma_ratio": 12.0,
           "bytes_per_update": nbytes, "bytes_basis": f"{SC_BYTES_PER_PARTICLE} B per particle + "
                                                     f"{SC_BYTES_PER_CELL} B per cell (compulsory HBM traffic)"}

    def make(mode, qscale=1.0):
        b = FFAG_Bunch(v, marcosize=1e13 / n * qscale, sc_grid_size=(*SC_GRID, 12.0), BunchType="Boris", device=dev)
        b.SEO_fi_axis, b.SEO_Ek_axis, b.SEO_r_matrix = seo["fi_axis"], seo["Ek_axis"], seo["r"]
        b.SEO_pr_matrix, b.SEO_perimeter = seo["pr"], seo["perimeter"]
        return b, SpaceCharge(b, hockney=(mode == "hockney"))

    for mode in ("periodic", "hockney"):
        b, sc = make(mode)
        for k in range(warmup):
            sc.update(first=(k == 0))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(sc.stream)
        for k in range(updates):
            sc.update(first=False)
        e1.record(sc.stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / updates
        out[f"{mode}_ms_per_update"] = ms
        out[f"{mode}_roofline"] = {"bound": "hbm", "achieved": nbytes / (ms * 1e-3) / 1e9, "peak": hbm_peak,
                                   "unit": "GB/s", "frac": nbytes / (ms * 1e-3) / 1e9 / hbm_peak}
        del sc, b

    sc_steps = STEPS_PER_TURN // 12

    def cycle(precision, nturns, qscale=1.0, with_sc=True):
        b, sc = make("hockney", qscale)
        pusher = Pusher(b, gp, "Boris", precision)
        clock = StepClock(0.0, dt, gp.Emap, "Boris", dev)
        clock.ensure(STEPS_PER_TURN * (nturns + 1))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(sc.stream)
        step = 0
        for k in range(nturns * 12):
            if with_sc:     # an update every 60 steps from step 0, as the step loop does
                sc.update(first=(k == 0))
            pusher.push(clock, step, sc_steps, sc_steps if with_sc else 0)
            step += sc_steps
        e1.record(sc.stream)
        torch.cuda.synchronize()
        alive = float((b.cols["surv"] == 1).float().mean().item())
        return e0.elapsed_time(e1), alive

    cycle("fp32c", 1)                   # warm-up
    ms32, _ = cycle("fp32c", turns)
    cycle("fp64", 1)                    # warm-up (the FP64 pusher's first particle order)
    ms64, _ = cycle("fp64", turns)
    out["cycle"] = "12 x (open-boundary update + 60 Boris FP32C steps) per turn"
    out["cycle_particle_turns_per_s"] = n * turns / (ms32 * 1e-3)
    out["cycle_fp64_particle_turns_per_s"] = n * turns / (ms64 * 1e-3)
    out["cycle_ms_per_turn"] = {"fp32c": ms32 / turns, "fp64": ms64 / turns}
    _, a1 = cycle("fp32c", 1)
    _, a3 = cycle("fp32c", 1, qscale=1e-3)
    _, a0 = cycle("fp32c", 1, with_sc=False)
    out["alive_fraction_after_one_turn"] = {"full_charge": a1, "charge_x1e-3": a3, "no_space_charge": a0}
    return out


def rk4_bench(gp, dt, dev, steps, warmup, flush, n=N_PARTICLES, seed=7, precision="fp64"):
    """c1 with the RK4 pusher (float64, or the FP32C field): the same
    lattice, RF and bunch (RK4 columns: f5 = total energy), 720 steps per
    turn, one turn per launch, L2 flushed and the bunch restored between
    launches (outside the events)."""
    import torch
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_ConversionTools
    from pyffa_b200.track import Pusher, StepClock, _EphemeralBunch
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek(synthetic.centred_bunch(n, seed=seed))
    v[:, 7] = 1.0
    v[:, 8] = 1.0
    b = _EphemeralBunch(v, "RK4", dev)
    pristine = {k: t.clone() for k, t in b.cols.items()}
    pu = Pusher(b, gp, "RK4", precision)
    clock = StepClock(0.0, dt, gp.Emap, "RK4", dev)
    clock.ensure(STEPS_PER_TURN * (warmup + steps + 1))
    stream = pu.stream

    def restore():
        for k, t in b.cols.items():
            t.copy_(pristine[k])

    for k in range(warmup):
        restore()
        pu.push(clock, k * STEPS_PER_TURN, STEPS_PER_TURN, 0)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        restore()
        flush.zero_()
        ev[k][0].record(stream)
        pu.push(clock, (warmup + k) * STEPS_PER_TURN, STEPS_PER_TURN, 0)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(bb) for a, bb in ev)
    return {"value": n / (ms * 1e-3), "unit": "particle-turns/s", "ms_per_turn": ms, "particles": n,
            "steps_per_turn": STEPS_PER_TURN, "launches": steps, "precision": precision}


def c1_accuracy_bench(gp, dt, dev, n=N_PARTICLES, turns=1000, tune_n=1024, seed=7):
    """c1's accuracy report: the c1 bunch tracked for 1000 turns with the RF
    on by the float64 Boris pusher (the reference for the errors), the FP32C
    Boris pusher and the float64 RK4 pusher, and by the float64 Boris pusher
    from every radius times 1 + 2^-24 (the dynamics' own response to a
    float32-sized input change); the RK4 pusher with the FP32C field beside
    them.  Coordinates and rms emittances are compared
    where the particles cross the azimuth half a turn from the bunch in the
    last turn; tunes (FFT, the reference's estimator) from 1000 turns of
    crossings of the first `tune_n` particles."""
    import tempfile
    import torch
    from pyffa_b200 import diagnostics as D
    from pyffa_b200 import synthetic
    from pyffa_b200.bunch import FFAG_Bunch
    from pyffa_b200.constants import E0_J, FFAG_ConversionTools
    from pyffa_b200.dump import Dumps, PositionDumpBunch
    from pyffa_b200.track import FFAG_RungeKutta
    p = synthetic.centred_bunch(n, seed=seed)
    conv = FFAG_ConversionTools()
    target = (np.pi + np.mean(p[:, 4])) % (2 * np.pi)
    nsteps = turns * STEPS_PER_TURN

    def run(solver, precision, m, window_turns):
        b = FFAG_Bunch(m, BunchType=solver, device=dev)
        d = PositionDumpBunch(np.rad2deg(target), (nsteps - window_turns * STEPS_PER_TURN - 0.05 * STEPS_PER_TURN) * dt,
                              (nsteps - 0.05 * STEPS_PER_TURN) * dt, save_folder=os.path.join(tempfile.mkdtemp(), "x"))
        dumps = Dumps()
        dumps.add_dump(d)
        lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
              "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": dumps}
        rk = FFAG_RungeKutta(precision=precision, verbose=False)
        getattr(rk, "rk4_solve_dt_bunch3_withSC" if solver == "RK4" else "rk4_solve_dt_bunch3_withSC_boris")(
            None, 0.0, b, gp, lp)
        torch.cuda.synchronize()
        return d.crossing_records, b.LocalBunch

    vb = conv.ConvertPrzek2Vrzek_boris(p)
    vr = conv.ConvertPrzek2Vrzek(p)
    vb32 = vb.copy()
    vb32[:, 0] *= 1 + 2.0 ** -24
    cases = {"fp64_boris": ("Boris", "fp64", vb), "fp32c_boris": ("Boris", "fp32c", vb),
             "fp32_boris": ("Boris", "fp32", vb),
             "fp64_rk4": ("RK4", "fp64", vr), "fp32c_rk4": ("RK4", "fp32c", vr),
             "fp64_boris_r_1_2e-24": ("Boris", "fp64", vb32)}
    last, tun, alive = {}, {}, {}
    for name, (solver, prec, m) in cases.items():
        t0 = time.perf_counter()
        rec, end = run(solver, prec, m.copy(), 0.9)
        last[name] = D.at_azimuth(rec, n, dt, solver, E0_J)
        alive[name] = int((end[:, 8] == 1).sum())
        rec_t, _ = run(solver, prec, m[:tune_n].copy(), turns)
        tun[name] = D.tunes(D.crossing_table(rec_t, tune_n, dt, solver, E0_J))
        last[name + "_s"] = time.perf_counter() - t0
    out = {"particles": n, "turns": turns, "steps_per_turn": STEPS_PER_TURN, "rf": "2 gaps, last-gap semantics",
           "vs": "fp64_boris", "tune_particles": tune_n, "alive": alive}
    for name in ("fp32c_boris", "fp32_boris", "fp64_rk4", "fp32c_rk4", "fp64_boris_r_1_2e-24"):
        e = D.azimuth_errors(last["fp64_boris"], last[name])
        dq = np.abs(tun[name] - tun["fp64_boris"])
        dq = np.minimum(dq, 1.0 - dq)
        ok = np.isfinite(dq).all(1)
        e["tune_max"] = [float(dq[ok, 0].max()), float(dq[ok, 1].max())] if ok.any() else None
        e["tune_rms"] = [float(np.sqrt(np.mean(dq[ok, 0] ** 2))), float(np.sqrt(np.mean(dq[ok, 1] ** 2)))] \
            if ok.any() else None
        e["wall_s"] = last[name + "_s"]
        out[name] = e
    q = tun["fp64_boris"]
    out["fp64_boris_tunes_median"] = [float(np.nanmedian(q[:, 0])), float(np.nanmedian(q[:, 1]))]
    return out


def mapgen_bench(dev, hbm_peak, reps=5):
    """z-Taylor map generation on the workloads' 1301 x 6000 grid, order 2
    (the reference's offline Generate_Bmaps_MultiProcess): device time of the
    build (CUDA events, tables resident in HBM), end-to-end time of the
    reference-facing call (numpy tables on the host), and the oracle port on
    a sample of rows, scaled to the whole map."""
    import torch
    from numpy.polynomial import Polynomial
    from oracle import mapgen as M
    from pyffa_b200 import mapgen as G
    from pyffa_b200 import synthetic
    B = synthetic.lattice_bmap()["Bmap"]
    B["SpiralAngle_deg"] = 20.0
    r, fi = G.map_axes(B)
    sfit = Polynomial.fit(r, G.calculate_s(r, 0.0, B["SpiralAngle_deg"]), 5)
    conv = G.BmapParams_to_ConvexParams(B)
    ak = B["coefficients_tupel"]
    plan = G.MapgenPlan(2, r, fi, conv, sfit, ak, device=dev)
    for _ in range(3):
        plan.run()
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        plan.run()
        b.record()
        torch.cuda.synchronize(dev)
        ms.append(a.elapsed_time(b))
    del plan
    t0 = time.perf_counter()
    G.Generate_Bmaps(2, r, fi, conv, sfit, ak)
    e2e_s = time.perf_counter() - t0
    rows = [0, 650]
    t0 = time.perf_counter()
    M.generate_bmaps(2, r[rows], fi, M.convex_params(B), sfit, ak)
    cpu_row_s = (time.perf_counter() - t0) / len(rows)
    written = 9 * len(r) * len(fi) * 8
    gpu_s = statistics.median(ms) / 1e3
    return {"grid": [len(r), len(fi)], "max_order": 2, "spiral_deg": 20.0,
            "gpu_ms": statistics.median(ms), "e2e_s": e2e_s,
            "hbm": {"bytes_written": written, "achieved_gbs": written / gpu_s / 1e9, "peak_gbs": hbm_peak,
                    "frac": written / gpu_s / 1e9 / hbm_peak},
            "cpu_port_s_per_map": cpu_row_s * len(r), "cpu_port_sample": f"{len(rows)} rows x {len(fi)} azimuths, "
                                                                        "1 thread, scaled to the map"}


def seo_scan_bench(dev, n_energies=256):
    """Batched closed-orbit and tune scan: 256 energies 300-600 MeV through the
    GPU closed-orbit search (all energies' azimuth tracks of an iteration in
    one launch), and the same search with the oracle's CPU tracker on a
    sample of energies, scaled."""
    import torch
    from oracle import oracle as O
    from pyffa_b200 import seo, synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical
    cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=0, AddNumricalMap=False)
    bm.UpdataConfig()
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    Ek = np.linspace(300.0, 600.0, n_energies)
    finder = seo.FFAG_SearchSEO(gp, device=dev)
    calls = {"n": 0}
    run = finder.tracker.run

    def counted(*a, **k):
        calls["n"] += 1
        return run(*a, **k)

    finder.tracker.run = counted
    finder.search(Ek[:4])          # warm-up
    torch.cuda.synchronize(dev)
    calls["n"] = 0
    t0 = time.perf_counter()
    res = finder.search(Ek)
    gpu_s = time.perf_counter() - t0
    sample = Ek[::64]
    cpu = seo.FFAG_SearchSEO(gp, tracker=O.ThetaTracker(gp.Bmap, gp.q))
    t0 = time.perf_counter()
    cpu.search(sample)
    cpu_s = (time.perf_counter() - t0) * len(Ek) / len(sample)
    return {"energies": n_energies, "Ek_MeV": [300.0, 600.0], "wall_s": gpu_s, "launches": calls["n"],
            "Qr_range": [float(res["table"][:, 2].min()), float(res["table"][:, 2].max())],
            "Qz_range": [float(res["table"][:, 3].min()), float(res["table"][:, 3].max())],
            "cpu_port_s_est": cpu_s, "cpu_port_threads": O.num_threads(),
            "cpu_port_sample": f"{len(sample)} of the energies with the oracle tracker, scaled"}


def coscan_bench(gp, dev, n_instances=256, turns=200, iterations=2, seed=0, steps_per_turn=2880):
    """Batched closed-orbit / tune scan (c3): 256 instances at energies
    300-600 MeV (linspace), ceil(exp(U(0, ln 4096))) particles each with
    0.5 mm Gaussian offsets, all in one bunch through the FP32C Boris pusher
    (RF off), 200 turns of the slowest instance per iteration, float64
    one-turn-map fit and fixed-point update per instance; the push's launch
    shape picked by the autotuner on the scan's bunch first; each iteration
    one push launch over all its steps, the kernel adding every crossing to
    its instance's normal equations (no crossing records); iteration 1
    direct, iteration 2 captured as a CUDA graph, later ones replays.  2880
    steps per
    turn of the fastest instance: at 720 the 2.8-degree D magnet gets five
    steps and the motion is not regular enough for a tune."""
    import torch
    from pyffa_b200 import coscan, synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_EField_new
    gp2 = FFAG_GlobalParameters()
    gp2.AddBMap(gp.Bmap)
    gp2.AddEMap(FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=False))
    E = np.linspace(300.0, 600.0, n_instances)
    counts = coscan.instance_counts(n_instances, 4096, seed)
    d = synthetic.design(300.0)
    k = float(gp.Bmap.k_value)
    scale = (synthetic.momentum(E) / synthetic.momentum(300.0)) ** (1 / (k + 1))
    r_sc = d["r0"] * scale
    scan = coscan.BatchedOrbitScan(gp2, E, counts, r_sc + 1e-4, np.full(n_instances, np.arctan(d["pr0"])),
                                   d["perimeter"] * scale, sigma=0.5e-3, turns=turns, seed=seed, device=dev,
                                   steps_per_turn=steps_per_turn)
    # iteration 1 direct, iteration 2 captured as a CUDA graph, then replays
    recs = [scan.iterate(graph=False)] + [scan.iterate(graph=True) for _ in range(iterations)]
    torch.cuda.synchronize(dev)
    pt = sum(r["particle_turns"] for r in recs)
    ms = sum(r["ms"] for r in recs)
    q = recs[-1]["tunes"]
    return {"value": pt / (ms * 1e-3), "unit": "particle-turns/s (sum over instances)",
            "particle_steps_per_s": scan.N * scan.steps * len(recs) / (ms * 1e-3),
            "instances": n_instances, "particles": scan.N, "turns_per_iteration": turns,
            "steps_per_iteration": scan.steps, "steps_per_turn_fastest": steps_per_turn, "iterations": len(recs),
            "ms_per_iteration": [r["ms"] for r in recs], "modes": [r["mode"] for r in recs],
            "push_launches_per_iteration": recs[-1]["launches"],
            "steps_per_launch": scan._dev_state.L,
            "accumulate": scan.accumulate,
            "fit_memory_mb": sum(t.numel() * t.element_size() for t in
                                 (scan._dev_state.sums, scan._dev_state.fit_last, scan._dev_state.fit_has,
                                  scan._dev_state.fit_inst)) / 1e6,
            "max_abs_dr_m": [r["max_abs_dr"] for r in recs],
            "orbit_vs_scaling_law_m": float(np.abs(scan.r - r_sc).max()),
            "Qr_frac_range": [float(np.nanmin(q[:, 0])), float(np.nanmax(q[:, 0]))],
            "Qz_frac_range": [float(np.nanmin(q[:, 1])), float(np.nanmax(q[:, 1]))],
            "padding_waste": scan.padding(), "valid_instances": int(recs[-1]["good"].sum()),
            "dtype": "f32c push, f64 fit and update",
            "graph": "iteration 1 direct; iteration 2 captured as one CUDA graph; iteration 3 a replay",
            "autotune": None if scan.tuning is None else
            {"shape": scan.tuning.report()["chosen"], "speedup_vs_default_shape": scan.tuning.speedup,
             "tune_steps": scan.tune_steps, "rtol": scan.tune_rtol, "candidates": _tune_rows(scan.tuning)}}


def _tune_rows(res):
    """Autotuner table, compact: [threads, register cap, warps per SM, ms,
    largest relative state difference from the default shape, accepted]."""
    return [[r["threads"], r["max_regs"], r.get("warps_per_sm"), round(r["ms"], 4), r.get("max_rel_diff"),
             r.get("accepted")] for r in res.rows]


# algorithmic flops of one map application: 5 inputs (the sixth is zero),
# two 256 x 256 hidden layers, 4 fitted outputs
LEARNED_FLOP_PER_MAP = 2 * (5 * 256 + 2 * 256 * 256 + 256 * 4)
# executed on the tensor cores (K = 16 layer-1 tile, N = 16 layer-4 tile)
LEARNED_MMA_FLOP_PER_MAP = 2 * (16 * 256 + 2 * 256 * 256 + 256 * 16)


def same_lattice_push(gp_l, phys, dev, turns=2, steps_per_turn=STEPS_PER_TURN):
    """The plain time-domain Boris pushers (FP64, FP32C) on the learned map's
    own lattice (analytic field, no z-Taylor map, no RF) and bunch (the
    learned map's states as Boris states at fi = 0), `steps_per_turn` steps
    of the 300 MeV design per launch.  The bunch spans 300-600 MeV, so a
    launch carries each particle through a different fraction of a turn: the
    particle-turns are counted from each particle's azimuth advance."""
    import torch
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_EField_new
    from pyffa_b200.learned import phys_to_boris
    from pyffa_b200.track import Pusher, StepClock, _EphemeralBunch
    gp2 = FFAG_GlobalParameters()
    gp2.AddBMap(gp_l.Bmap)
    gp2.AddEMap(FFAG_EField_new(synthetic.emap_file(os.path.join(tempfile.mkdtemp(), "emap.txt")), EnableFlag=False))
    m = phys_to_boris(phys)
    spt = int(steps_per_turn)
    dt = synthetic.design_dt(300.0, spt)
    out = {"particles": m.shape[0], "launches": turns, "steps_per_launch": spt,
           "lattice": "the learned map's: analytic field, no z-Taylor map, no RF"}
    for prec in ("fp64", "fp32c"):
        b = _EphemeralBunch(m, "Boris", dev)
        pu = Pusher(b, gp2, "Boris", prec)
        clock = StepClock(0.0, dt, gp2.Emap, "Boris", dev)
        clock.ensure(spt * (turns + 2))
        pu.push(clock, 0, spt, 0)
        torch.cuda.synchronize()
        fi0 = b.cols["fi"].clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(pu.stream)
        for k in range(turns):
            pu.push(clock, (k + 1) * spt, spt, 0)
        e1.record(pu.stream)
        torch.cuda.synchronize()
        pturns = float(((b.cols["fi"] - fi0) / (2 * np.pi)).sum().item())
        ms = e0.elapsed_time(e1)
        out[prec] = {"value": pturns / (ms * 1e-3), "unit": "particle-turns/s", "ms_per_launch": ms / turns,
                     "particle_turns": pturns}
        del b, pu
        torch.cuda.empty_cache()
    return out, gp2, dt


LEARNED_STEPS_PER_TURN = 2880     # the learned map's plain tracker: Boris, 2880 steps per 300 MeV turn


def learned_bench(dev, fp64_value, fp32c_value, samples=20_000_000, epochs=8, n=10_000_000, turns_per_step=50,
                  steps=10, check_n=512, check_turns=1000):
    """Learned sector map: train on `samples` one-sector crossings of the
    plain FP32C time-domain Boris pusher (2880 steps per 300 MeV turn;
    300-600 MeV, amplitudes up to 10 mm / 5 mrad, uniform in normalised
    phase space), then track an n-particle bunch with audits every 50 turns
    on 1% of the states against the same pusher (one step = 50 turns), and
    compare a check bunch over 1000 turns with the FP64 Boris pusher at the
    same step (and with the azimuth-domain RK4 tracker)."""
    import torch
    from pyffa_b200 import learned, synthetic
    from pyffa_b200.constants import FFAG_ConversionTools, FFAG_GlobalParameters
    from pyffa_b200.fields import FFAG_Bfield_analytical
    cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
    bm = FFAG_Bfield_analytical(config=cfg, max_order=0, AddNumricalMap=False)
    bm.UpdataConfig()
    gp = FFAG_GlobalParameters()
    gp.AddBMap(bm)
    dt_td = synthetic.design_dt(300.0, LEARNED_STEPS_PER_TURN)
    tracker = learned.TimeDomainSectorTracker(gp, dt_td, "fp32c", device=dev)      # data, audits, fall-back
    t64 = learned.TimeDomainSectorTracker(gp, dt_td, "fp64", device=dev)          # frame and reference
    rk4 = learned.SectorTracker(gp.Bmap, gp.q, steps_per_sector=128, device=dev)  # azimuth-domain check
    d0 = synthetic.design(300.0)
    conv = FFAG_ConversionTools()
    nodes = np.cos(np.pi * (np.arange(17) + 0.5) / 17)[::-1]
    P = conv.Ek2P(450.0 + 150.0 * nodes)
    r_guess = d0["r0"] * (P / conv.Ek2P(300.0)) ** (1 / (cfg["Bmap"]["coefficients_tupel"][1] + 1))
    frame = learned.SectorFrame.build(t64, (300.0, 600.0), (10e-3, 5e-3), r_guess=r_guess, pr_guess=d0["pr0"])
    t0 = time.perf_counter()
    X, T = learned.make_dataset(frame, tracker, samples, seed=1)
    Xv, Tv = learned.make_dataset(frame, tracker, 1 << 16, seed=2)
    torch.cuda.synchronize(dev)
    t_data = time.perf_counter() - t0
    p = torch.from_numpy(learned.init_params(3)).to(dev)
    t0 = time.perf_counter()
    _, tr = learned.train(p, X, T, epochs=epochs, batch=8192, lr=2e-3, time_limit=90.0)
    torch.cuda.synchronize(dev)
    t_train = time.perf_counter() - t0
    mse = learned.evaluate(p, Xv, Tv)
    del X, T
    torch.cuda.empty_cache()

    # the n-particle bunch: Gaussian (sigma 0.3) inside radius 0.9, energies across the range
    def bunch(m, seed):
        rng = np.random.default_rng(seed)
        s = np.zeros((m, 5))
        s[:, :4] = 0.3 * rng.standard_normal((m, 4))
        for j in (0, 2):
            r = np.hypot(s[:, j], s[:, j + 1])
            s[:, j:j + 2] *= np.minimum(1.0, 0.9 / np.maximum(r, 1e-12))[:, None]
        s[:, 4] = rng.uniform(-0.9, 0.9, m)
        st = torch.from_numpy(s).to(dev)
        Pm = torch.as_tensor(frame.P_of_Ek(frame.Ek_of(s[:, 4])), device=dev)
        return torch.cat([frame.to_phys(st, st[:, 4]), Pm[:, None]], 1)

    lm = learned.LearnedSectorMap(frame, tracker, p, audit_every=50, audit_frac=0.01, audit_tol=1e-5)
    phys = bunch(n, 5)
    lm.track(phys, turns_per_step)                      # warm-up
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    launches0 = lm.launches
    audits = []
    for k in range(steps):
        ev[k][0].record()
        res = lm.track(phys, turns_per_step)
        ev[k][1].record()
        audits += res["audits"]
    torch.cuda.synchronize(dev)
    mlp_launches = (lm.launches - launches0) // max(steps, 1)
    ms = [a.elapsed_time(b) for a, b in ev]
    value = n * turns_per_step * steps / (sum(ms) * 1e-3)
    # the inference kernel alone: 50 turns of maps in one launch, states resident
    st = torch.zeros((n, 8), dtype=torch.float32, device=dev)
    st[:, :5] = frame.to_norm(phys).float()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lm.apply(st, 12)
    e0.record()
    lm.apply(st, turns_per_step * 12)
    e1.record()
    torch.cuda.synchronize(dev)
    k_s = e0.elapsed_time(e1) * 1e-3
    maps = n * turns_per_step * 12
    try:
        mp = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
        peaks = {"burst": mp["bf16_tflops"], "sustained": mp["bf16_tflops_sustained"],
                 "source": "MEASURED_PEAKS.json bf16 cuBLAS (of measured; sustained: seconds-long launch)"}
    except Exception:
        peaks = {"burst": 1590.0, "sustained": 1400.0,
                 "source": "fallback (MEASURED_PEAKS.json absent): 1.59 PF/s burst, 1.4 sustained"}
    ach = LEARNED_FLOP_PER_MAP * maps / k_s / 1e12
    # the plain time-domain pushers on the same lattice and bunch: at the
    # learned map's own step (the tracker it replaces) and at c1's
    same, _, _ = same_lattice_push(gp, phys, dev, steps_per_turn=LEARNED_STEPS_PER_TURN)
    same["speedup_vs_fp64_same_lattice"] = value / same["fp64"]["value"]
    same["speedup_vs_fp32c_same_lattice"] = value / same["fp32c"]["value"]
    same720, _, _ = same_lattice_push(gp, phys, dev, steps_per_turn=STEPS_PER_TURN)
    same["at_720_steps_per_turn"] = {k: same720[k] for k in ("fp64", "fp32c")}
    same["at_720_steps_per_turn"]["speedup_vs_fp64"] = value / same720["fp64"]["value"]
    same["at_720_steps_per_turn"]["speedup_vs_fp32c"] = value / same720["fp32c"]["value"]
    del phys
    torch.cuda.empty_cache()
    # accuracy: a check bunch over 1000 turns against the FP64 Boris pusher
    # at the same step, and against the azimuth-domain RK4 tracker
    cb = bunch(check_n, 4)
    ref = learned.plain_track(frame, t64, cb, check_turns, record=True)
    got = learned.LearnedSectorMap(frame, tracker, p, audit_every=50, audit_frac=0.01,
                                   audit_tol=1e-5).track(cb, check_turns, record=True)
    dq = np.abs(learned.tunes(got["record"]) - learned.tunes(ref["record"]))
    de = np.abs(learned.betatron_emittance(frame, got["record"][-1]) /
                learned.betatron_emittance(frame, ref["record"][-1]) - 1)
    rr = learned.plain_track(frame, rk4, cb, check_turns, record=True)
    qr = learned.tunes(rr["record"])
    er = learned.betatron_emittance(frame, rr["record"][-1])
    dqr = np.abs(learned.tunes(got["record"]) - qr)
    der = np.abs(learned.betatron_emittance(frame, got["record"][-1]) / er - 1)
    dqbr = np.abs(learned.tunes(ref["record"]) - qr)
    debr = np.abs(learned.betatron_emittance(frame, ref["record"][-1]) / er - 1)
    return {
        "value": value, "unit": "particle-turns/s",
        "speedup_vs_fp64": value / fp64_value if fp64_value else None,
        "speedup_vs_fp32c": value / fp32c_value if fp32c_value else None,
        "ms_per_step": statistics.mean(ms), "turns_per_step": turns_per_step, "particles": n,
        "audit": {"every_turns": 50, "fraction": 0.01, "tol": 1e-5,
                  "sampled": int(sum(a[1] for a in audits)), "failed": int(sum(a[2] for a in audits)),
                  "max_error": max((a[3] for a in audits), default=None)},
        "plain_fallback_states": int(res["plain"].sum()),
        "kernel": {"maps_per_launch": turns_per_step * 12, "s": k_s, "particle_turns_per_s": n * turns_per_step / k_s,
                   "roofline": {"bound": "tensor", "achieved": ach, "unit": "TFLOP/s",
                                "peak": peaks["sustained"], "frac": ach / peaks["sustained"],
                                "peak_burst": peaks["burst"], "frac_of_burst": ach / peaks["burst"],
                                "flop_per_map": LEARNED_FLOP_PER_MAP,
                                "mma_flop_per_map": LEARNED_MMA_FLOP_PER_MAP,
                                "peak_source": peaks["source"]}},
        "plain_tracker": f"FP32C time-domain Boris, {LEARNED_STEPS_PER_TURN} steps per 300 MeV turn",
        "accuracy": {"check_bunch": check_n, "turns": check_turns, "tune_error_max": float(dq.max()),
                     "tune_error_rms": float(np.sqrt(np.mean(dq ** 2))),
                     "emittance_error_max": float(de.max()),
                     "vs": f"FP64 time-domain Boris, {LEARNED_STEPS_PER_TURN} steps per 300 MeV turn",
                     "vs_azimuth_rk4": {"tune_error_max": float(dqr.max()), "emittance_error_max": float(der.max()),
                                        "boris_vs_rk4_tune_max": float(dqbr.max()),
                                        "boris_vs_rk4_emittance_max": float(debr.max()),
                                        "rk4": "FP64 azimuth-domain RK4, 128 steps per sector"}},
        "same_lattice": same,
        "training": {"samples": samples, "epochs": epochs, "batch": 8192, "s": t_train, "data_s": t_data,
                     "steps": tr.t, "samples_per_s": tr.t * 8192 / t_train, "validation_mse": mse,
                     "residual_scale": tr.out_scale},
        "mlp_launches_per_step": mlp_launches,
        "dtype": "bf16 tensor-core hidden layers, f32 accumulation, f32 skip and state",
    }


def bench_config(n, precision, world):
    """The workload both arms report (identical dicts)."""
    return {"workload": "c1: 12-sector FFAG, 300 MeV, 1301x6000 map z-Taylor order 2, 2 RF gaps "
                        "(last-gap semantics), Boris, 720 steps/turn, 1 turn per step",
            "particles_per_gpu": n, "steps_per_turn": STEPS_PER_TURN, "precision": precision,
            "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{world}"}


METRIC = "particle-turns/s (Boris FP64, 1e5-particle bunch, 2 RF gaps, z-Taylor order 2)"


def run_reference(args):
    """--impl reference: the reference's algorithm on the host cores (the
    oracle's C port, every thread; on one host it runs at 1.07x the
    reference's own Numba path, oracle/time_reference_numba.py), on the same
    bunch as the GPU arm; each step a bounded sample of one turn: the whole
    bunch through REF_SAMPLE_STEPS of the turn's 720 steps, scaled."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    gp, v, dt = workload(n=args.n)
    from oracle import oracle as O
    O.build()
    S = O.Setup(gp.Bmap, gp.Emap, gp)
    O.boris_step(S, np.ascontiguousarray(v[:64].copy()), 0.0, dt)    # warm the library
    times = []
    for k in range(args.warmup + args.steps):
        m = np.ascontiguousarray(v.copy())
        t0 = time.perf_counter()
        O.track(S, "Boris", m, 0.0, dt, REF_SAMPLE_STEPS)
        el = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(el)
    n = v.shape[0]
    per_turn_s = sum(times) / len(times) * STEPS_PER_TURN / REF_SAMPLE_STEPS
    val = n / per_turn_s
    sample = (f"{n} particles (the GPU arm's bunch) x {REF_SAMPLE_STEPS} of the {STEPS_PER_TURN} steps of a turn "
              f"per step, scaled to a turn")
    line = {"metric": METRIC, "value": val, "unit": "particle-turns/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per_turn_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 6D Gaussian bunch, analytic lattice)",
            "config": bench_config(n, "fp64", args.gpus),
            "cpu_baseline": {"value": val, "unit": "particle-turns/s", "cores": O.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": val, "unit": "particle-turns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    from pyffa_b200.track import MatrixTracker, Pusher, StepClock, _EphemeralBunch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    gp, v, dt = workload(seed=7 + rank, n=args.n)
    n = v.shape[0]
    total_steps = STEPS_PER_TURN * (args.warmup + args.steps + 1)
    b = _EphemeralBunch(v, "Boris", dev)
    pristine = {k: t.clone() for k, t in b.cols.items()}
    pusher = Pusher(b, gp, "Boris", args.precision)
    clock = StepClock(0.0, dt, gp.Emap, "Boris", dev)
    clock.ensure(total_steps)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = pusher.stream

    def restore():
        # every timed step starts from the same bunch (not timed)
        for k, t in b.cols.items():
            t.copy_(pristine[k])

    def timed_turns(pu, steps):
        """CUDA-event time of each one-turn launch, L2 flushed and the bunch
        restored before each (outside the events)."""
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            restore()
            flush.zero_()
            ev[k][0].record(stream)
            pu.push(clock, (args.warmup + k) * STEPS_PER_TURN, STEPS_PER_TURN, 0)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(bb) for a, bb in ev]

    for k in range(args.warmup):
        restore()
        pusher.push(clock, k * STEPS_PER_TURN, STEPS_PER_TURN, 0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    b.status.zero_()
    with ClockSampler(local) as cs:
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        launch_ms = timed_turns(pusher, args.steps)
        if world > 1:
            dist.barrier()
    t_ms = sum(launch_ms)
    t = torch.tensor([t_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_ms = float(t.item())
    status = b.status.cpu().numpy()
    value = n * world * args.steps / (t_ms * 1e-3)

    # the same FP64 kernel on a 1e6-particle bunch (fills the GPU: the 1e5
    # bunch gives 21 warps per SM), 10 one-turn launches
    large = None
    if not args.no_large and args.n == N_PARTICLES and args.precision == "fp64" and world == 1:
        from pyffa_b200 import synthetic
        from pyffa_b200.constants import FFAG_ConversionTools
        vl = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(synthetic.centred_bunch(1_000_000, seed=17))
        vl[:, 7] = 1.0
        vl[:, 8] = 1.0
        bl = _EphemeralBunch(vl, "Boris", dev)
        pul = Pusher(bl, gp, "Boris", "fp64")
        pul.push(clock, 0, STEPS_PER_TURN, 0)
        torch.cuda.synchronize()
        el = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(10)]
        for k in range(10):
            el[k][0].record(stream)
            pul.push(clock, (k + 1) * STEPS_PER_TURN, STEPS_PER_TURN, 0)
            el[k][1].record(stream)
        torch.cuda.synchronize()
        lms = statistics.mean(a.elapsed_time(bb) for a, bb in el)
        large = {"particles": 1_000_000, "value": 1_000_000 / (lms * 1e-3), "unit": "particle-turns/s",
                 "ms_per_turn": lms, "fp64_tflops": FP64_FLOP_PER_PARTICLE_STEP * 1e6 * STEPS_PER_TURN / (lms * 1e-3) / 1e12}
        del bl, pul

    # the compensated float32 pusher on the same workload
    fp32c = None
    if args.precision == "fp64" and not args.no_fp32c:
        pu32 = Pusher(b, gp, "Boris", "fp32c")
        for k in range(args.warmup):
            restore()
            pu32.push(clock, k * STEPS_PER_TURN, STEPS_PER_TURN, 0)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms32 = timed_turns(pu32, args.steps)
        t32 = torch.tensor([sum(ms32)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t32, op=dist.ReduceOp.MAX)
        v32 = n * world * args.steps / (float(t32.item()) * 1e-3)
        fp32c = {"value": v32, "unit": "particle-turns/s", "ms_per_step": float(t32.item()) / args.steps,
                 "speedup_vs_fp64": v32 / value,
                 "dtype": "f32 field exponentials and map lookup, f64 push and state"}
        # the launch-shape autotuner on this bunch (one-turn launches); the
        # chosen shape timed like the default one
        from pyffa_b200 import autotune
        tune = autotune.tune_push(pu32, clock, args.warmup * STEPS_PER_TURN, STEPS_PER_TURN, reset=restore)
        if world > 1:    # every rank times rank 0's choice (the same collectives on every rank)
            choice = torch.tensor(list(tune.best), dtype=torch.int64, device=dev)
            dist.broadcast(choice, 0)
            tune.best = (int(choice[0].item()), int(choice[1].item()))
            tune.best_ms = next(r["ms"] for r in tune.rows if r["shape"] == tune.best)
        tuned = {"shape": tune.report()["chosen"], "tuner_speedup": tune.speedup,
                 "candidates": _tune_rows(tune)}
        if tune.best != (0, 0):
            pu32.shape = tune.best
            mst = timed_turns(pu32, args.steps)
            tt = torch.tensor([sum(mst)], dtype=torch.float64, device=dev)
            if world > 1:
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            vt = n * world * args.steps / (float(tt.item()) * 1e-3)
            pu32.shape = (0, 0)
        else:
            vt = v32
        tuned.update({"value": vt, "speedup_vs_fp64": vt / value})
        fp32c["autotuned"] = tuned
        # the float32 pusher (float32 push, float64 accumulation of r, fi, z)
        pu32f = Pusher(b, gp, "Boris", "fp32")
        for k in range(args.warmup):
            restore()
            pu32f.push(clock, k * STEPS_PER_TURN, STEPS_PER_TURN, 0)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        msf = timed_turns(pu32f, args.steps)
        tf = torch.tensor([sum(msf)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(tf, op=dist.ReduceOp.MAX)
        vf = n * world * args.steps / (float(tf.item()) * 1e-3)
        fp32c["fp32_push"] = {"value": vf, "unit": "particle-turns/s", "ms_per_step": float(tf.item()) / args.steps,
                              "speedup_vs_fp64": vf / value,
                              "dtype": "f32 field and push, f64 accumulation of r, fi, z and the RF phase"}
    clocks = cs.summary()

    # end to end through the host-buffer API: host matrix in, one turn, host matrix out
    e2e = None
    if not args.no_e2e:
        mt = MatrixTracker(n, gp, "Boris", args.precision, device=dev)
        mt.bind_clock(0.0, dt, total_steps)
        # two pinned host matrices used in turn: each call reads one and
        # writes the other (the caller's buffers; no host-side copy between)
        hb = [torch.from_numpy(v.copy()).pin_memory(), torch.empty((n, 16), dtype=torch.float64).pin_memory()]
        for k in range(args.warmup):
            mt.run(hb[k % 2], hb[(k + 1) % 2], k * STEPS_PER_TURN, STEPS_PER_TURN)
            mt.pusher.stream.synchronize()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(mt.pusher.stream)
        for k in range(args.steps):
            j = args.warmup + k
            mt.run(hb[j % 2], hb[(j + 1) % 2], j * STEPS_PER_TURN, STEPS_PER_TURN)
            mt.pusher.stream.synchronize()
        e1.record(mt.pusher.stream)
        torch.cuda.synchronize()
        te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e = {"value": n * world * args.steps / (float(te.item()) * 1e-3), "unit": "particle-turns/s",
               "h2d_bytes_per_step": int(n * 16 * 8), "d2h_bytes_per_step": int(n * 16 * 8)}

    if rank == 0:
        peak64 = fp64_peak_tflops(local)
        if large is not None:
            large["fp64_frac"] = large["fp64_tflops"] / peak64
        if fp32c is not None:
            peak32 = fp32_peak_tflops(local)
            fp32c["fma_peaks_tflops"] = {"fp64": peak64, "fp32": peak32, "fp32_over_fp64": peak32 / peak64,
                                         "source": "measured live: FMA probe kernels (libffa_probe.so)"}
        avg_launch_s = (t_ms / args.steps) * 1e-3
        pstep = n * STEPS_PER_TURN
        roof = {"bound": "fp64", "unit": "TFLOP/s", "peak": peak64,
                "peak_source": "measured live: float64 FMA probe kernel (libffa_probe.so)"}
        ach = FP64_FLOP_PER_PARTICLE_STEP * pstep / avg_launch_s / 1e12
        ach_x = FP64_EXEC_FLOP_PER_PARTICLE_STEP * pstep / avg_launch_s / 1e12
        roof.update({"achieved": ach, "frac": ach / peak64,
                     "flop_per_particle_step": FP64_FLOP_PER_PARTICLE_STEP, "flop_basis": "algorithmic",
                     "executed": {"flop_per_particle_step": FP64_EXEC_FLOP_PER_PARTICLE_STEP,
                                  "achieved": ach_x, "frac": ach_x / peak64}})
        hbm_peak = None
        try:
            hbm_peak = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))["hbm_gbs"]
        except Exception:
            hbm_peak = 6650.0
        hbm_ach = STATE_BYTES_PER_PARTICLE * n / avg_launch_s / 1e9
        roof["hbm"] = {"bound": "hbm", "achieved": hbm_ach, "peak": hbm_peak, "unit": "GB/s",
                       "frac": hbm_ach / hbm_peak, "algorithmic_bytes_per_launch": STATE_BYTES_PER_PARTICLE * n,
                       "traffic": None}
        roof["traffic"] = BORIS_TRAFFIC_PER_LAUNCH if args.n == N_PARTICLES and args.precision == "fp64" else None
        roof["hbm"]["traffic"] = roof["traffic"]
        # the CPU baseline and the other workloads' legs at N = 1 only: with
        # more ranks they would hold every GPU while the others wait
        solo = world == 1
        cpu = None
        if not args.no_cpu_baseline and solo:
            cpu = cpu_baseline(gp, v, dt)
        sc = None
        if not args.no_sc and solo:
            sc = sc_bench(gp, dt, dev, hbm_peak)
        rk4 = None
        if not args.no_rk4 and solo:
            rk4 = rk4_bench(gp, dt, dev, min(args.steps, 10), args.warmup, flush)
            rk4["fp32c"] = rk4_bench(gp, dt, dev, min(args.steps, 10), args.warmup, flush, precision="fp32c")
            rk4["fp32c"]["speedup_vs_fp64_rk4"] = rk4["fp32c"]["value"] / rk4["value"]
            ach = RK4_FLOP_PER_PARTICLE_STEP * N_PARTICLES * STEPS_PER_TURN / (rk4["ms_per_turn"] * 1e-3) / 1e12
            rk4["roofline"] = {"bound": "fp64", "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                               "frac": ach / peak64, "flop_per_particle_step": RK4_FLOP_PER_PARTICLE_STEP,
                               "flop_basis": "algorithmic",
                               "peak_source": "measured live: float64 FMA probe kernel (libffa_probe.so)"}
        acc = None
        if not args.no_accuracy and solo:
            acc = c1_accuracy_bench(gp, dt, dev)
        mg = None
        if not args.no_mapgen and solo:
            mg = mapgen_bench(dev, hbm_peak)
        scan = None
        if not args.no_scan and solo:
            scan = seo_scan_bench(dev)
        csp = None
        if not args.no_coscan and solo:
            csp = coscan_bench(gp, dev)
        lrn = None
        if not args.no_learned and solo:
            lrn = learned_bench(dev, value / world, fp32c["value"] / world if fp32c else None,
                                samples=args.learned_samples, epochs=args.learned_epochs, n=args.learned_n)
        line = {
            "metric": METRIC,
            "value": value, "unit": "particle-turns/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32c",
            "data": "synthetic (seeded 6D Gaussian bunch, analytic lattice)",
            "config": bench_config(n, args.precision, world),
            "gpu_launches": args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks,
            "status": {"lost": int(status[0]), "nan": int(status[1]), "out_of_map": int(status[2])},
            "space_charge": sc,
            "rk4": rk4,
            "c1_accuracy": acc,
            "fp32c": fp32c,
            "mapgen": mg,
            "co_scan": scan,
            "learned_map": lrn,
            "co_scan_particles": csp,
            "fp64_1e6_particles": large,
            "launch_ms": {"mean": statistics.mean(launch_ms), "min": min(launch_ms), "max": max(launch_ms)},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
