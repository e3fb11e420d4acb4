"""Times the reference's own CPU path for the c1 workload next to the oracle's
C port, on the same host and the same particles.

The reference (PyFFA, Python + Numba) is imported from its checkout through
the single-rank stand-ins in tests/golden/shims (mpi4py, pyfftw,
matplotlib), the c1 lattice is written in its own Bmap folder format (full
1301 x 6000 map, z-Taylor order 2), and its step function
FFAG_RungeKutta.Boris_solve (src/FFAG_track.py:948-1049) is called step by
step on the c1 bunch (seeded 6D Gaussian, the same seed as the benchmark)
with Numba's thread pool at every host core (numba.set_num_threads;
main_track forces 1, examples/main_track.py:5-6).  The oracle's C port
(oracle/ffa_oracle.c, OpenMP, every host core) then tracks the same
particles over the same steps.  One JSON line: particle-steps/s and
particle-turns/s of both, the host's core count and CPU model.

With --c3, it times instead the reference's closed-orbit and tune search per
energy (FFAG_SearchSEO: SearchSEOUsingInitialEkVect + the one-turn track +
GetQrQz, src/FFAG_track.py:1245-1371 and 1441-1481) on the scan's lattice at
a few energies of 300-600 MeV, and extrapolates to the 256-energy scan.

Test infrastructure: needs the reference checkout (--ref PATH or
PYFFA_REFERENCE) and numba; it is not part of the library.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)

STEPS_PER_TURN = 720


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor()


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--ref", default=os.environ.get("PYFFA_REFERENCE"))
    ap.add_argument("--n", type=int, default=100_000)
    ap.add_argument("--steps", type=int, default=144)
    ap.add_argument("--c3", action="store_true")
    args = ap.parse_args()
    if not args.ref:
        ap.error("the reference checkout is required: --ref PATH or PYFFA_REFERENCE=PATH")
    if args.c3:
        return time_c3(args)
    sys.path.insert(0, os.path.join(REPO, "tests", "golden", "shims"))
    sys.path.insert(0, os.path.join(args.ref, "src"))
    import numba
    numba.set_num_threads(os.cpu_count())
    import FFAG_track
    from FFAG_Bunch import FFAG_Bunch
    from FFAG_Field import FFAG_Bfield_analytical, FFAG_BField_Error, FFAG_EField_new
    from FFAG_ParasAndConversion import FFAG_ConversionTools, FFAG_GlobalParameters

    from oracle import oracle as O
    from pyffa_b200 import synthetic
    from pyffa_b200.constants import FFAG_GlobalParameters as GP
    from pyffa_b200.fields import FFAG_Bfield_analytical as BA
    from pyffa_b200.fields import FFAG_EField_new as EN

    with tempfile.TemporaryDirectory() as tmp:
        cfg_path = synthetic.write_bmap_folder(os.path.join(tmp, "bmap"), 2)
        emap_path = synthetic.emap_file(os.path.join(tmp, "emap.txt"))
        gp = FFAG_GlobalParameters()
        gp.AddBMap(FFAG_Bfield_analytical(cfg_path, 2))
        gp.AddEMap(FFAG_EField_new(emap_path, True))
        gp.AddBHarmonics(FFAG_BField_Error([], False))
        gp.AddAperture(7.5, 9.5, -0.1, 0.1)
        p = synthetic.centred_bunch(args.n, seed=7)
        v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
        v[:, 7] = 1.0
        v[:, 8] = 1.0
        dt = synthetic.design_dt(300.0, STEPS_PER_TURN)

        def make(mat):
            return FFAG_Bunch(mat.copy(), BunchType="Boris")

        def step(b, t):
            FFAG_track.FFAG_RungeKutta().Boris_solve(
                t, b.LocalBunch, dt,
                b.Malloc_x_cart, b.Malloc_y_cart, b.Malloc_z_cart,
                b.Malloc_vx_cart, b.Malloc_vy_cart, b.Malloc_vz_cart,
                b.Malloc_Ex_cart, b.Malloc_Ey_cart, b.Malloc_Ez_cart,
                b.Malloc_Bx_cart, b.Malloc_By_cart, b.Malloc_Bz_cart,
                b.Malloc_RF_phase, b.Malloc_mod_fi,
                b.Malloc_Bz_interp, b.Malloc_Br_interp, b.Malloc_Bf_interp,
                b.Malloc_Ez_interp, b.Malloc_Er_interp, b.Malloc_Ef_interp,
                b.Step_SurviveFlag, b.Malloc_RF_shift,
                b.SurvivedNum_Local, b.LostNum_Local, gp)

        warm = make(v[:256])
        step(warm, 0.0)                        # Numba compiles here
        b = make(v)
        t = 0.0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step(b, t)
            t = t + dt
        ref_s = time.perf_counter() - t0
        ref_out = b.LocalBunch.copy()

        # the oracle port on the same particles and steps
        cfg = synthetic.lattice_bmap()
        gpo = GP()
        gpo.AddBMap(BA(config=cfg, max_order=2, stacks=synthetic.taylor_stacks(cfg, 2)))
        gpo.AddEMap(EN(emap_path, EnableFlag=True))
        gpo.AddAperture(7.5, 9.5, -0.1, 0.1)
        O.build()
        S = O.Setup(gpo.Bmap, gpo.Emap, gpo)
        m = np.ascontiguousarray(v.copy())
        O.boris_step(S, m[:64].copy(), 0.0, dt)
        t0 = time.perf_counter()
        O.track(S, "Boris", m, 0.0, dt, args.steps)
        port_s = time.perf_counter() - t0
    alive = ref_out[:, 8] == 1
    dr = np.abs(m[alive, 0] - ref_out[alive, 0]) / ref_out[alive, 0]
    ps = args.n * args.steps
    print(json.dumps({
        "workload": "c1 Boris fp64: 1301x6000 map, z-Taylor order 2, 2 RF gaps, 720 steps/turn",
        "particles": args.n, "steps": args.steps, "cores": os.cpu_count(), "cpu": cpu_model(),
        "reference_numba": {"s": ref_s, "particle_steps_per_s": ps / ref_s,
                            "particle_turns_per_s": ps / ref_s / STEPS_PER_TURN,
                            "numba": numba.__version__, "threads": numba.get_num_threads()},
        "oracle_port": {"s": port_s, "particle_steps_per_s": ps / port_s,
                        "particle_turns_per_s": ps / port_s / STEPS_PER_TURN, "threads": O.num_threads()},
        "port_over_reference": ref_s / port_s,
        "port_vs_reference_max_rel_r": float(dr.max()),
    }))


def time_c3(args, energies=(300.0, 400.0, 500.0, 600.0), n_scan=256):
    sys.path.insert(0, os.path.join(REPO, "tests", "golden", "shims"))
    sys.path.insert(0, os.path.join(args.ref, "src"))
    import numba
    numba.set_num_threads(os.cpu_count())
    from FFAG_Field import FFAG_Bfield_analytical, FFAG_BField_Error
    from FFAG_ParasAndConversion import FFAG_GlobalParameters
    from FFAG_track import FFAG_SearchSEO

    from pyffa_b200 import synthetic
    with tempfile.TemporaryDirectory() as tmp:
        cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
        cfg["config"]["folder"] = tmp
        path = os.path.join(tmp, "config_Bmap.json")
        with open(path, "w") as f:
            json.dump(cfg, f)
        FFAG_Bfield_analytical(path, 0, AddNumricalMap=False).UpdataConfig()   # as main_SEO does
        gp = FFAG_GlobalParameters()
        gp.AddBMap(FFAG_Bfield_analytical(path, 0, AddNumricalMap=False))
        gp.AddBHarmonics(FFAG_BField_Error([], False))
        finder = FFAG_SearchSEO(gp)
        per = []
        tunes = []
        for k, Ek in enumerate(energies):
            t0 = time.perf_counter()
            r0, pr0, _ = finder.SearchSEOUsingInitialEkVect(Ek, 0.001, 0.0, verbose=False)
            finder.TrackAParticle(r0, pr0, Ek, np.pi * 2, 0.001)
            Qr, Qz, *_ = finder.GetQrQz(r0, pr0, Ek, 0.001)
            el = time.perf_counter() - t0
            if k > 0 or len(energies) == 1:      # the first includes Numba's compilation
                per.append(el)
            tunes.append([float(Qr), float(Qz)])
    s_per = sum(per) / len(per)
    print(json.dumps({"workload": "c3 closed-orbit / tune search per energy, the scan's lattice (analytic field)",
                      "energies_timed": list(energies[1:]), "s_per_energy": s_per,
                      "scan_energies": n_scan, "scan_s_estimate": s_per * n_scan,
                      "tunes": tunes, "cores": os.cpu_count(), "cpu": cpu_model(),
                      "numba_threads": numba.get_num_threads()}))


if __name__ == "__main__":
    main()
