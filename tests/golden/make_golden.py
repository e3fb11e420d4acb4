"""Generates the golden vectors in tests/golden/ by running the reference
tracker (PyFFA, pure Python + Numba) on seeded synthetic inputs.

Run in the development container, where the reference source is available:
    python tests/golden/make_golden.py --ref REFERENCE_CHECKOUT              # tracking
    python tests/golden/make_golden.py --crossing --ref REFERENCE_CHECKOUT   # crossing dumps
    python tests/golden/make_golden.py --mapgen --ref REFERENCE_CHECKOUT     # z-Taylor maps
    python tests/golden/make_golden.py --seo --ref REFERENCE_CHECKOUT        # closed orbits
    python tests/golden/make_golden.py --bunch --ref REFERENCE_CHECKOUT      # injected bunches
    python tests/golden/make_golden.py --harmonics --ref REFERENCE_CHECKOUT  # field-error harmonics
    python tests/golden/make_golden.py --spiral --ref REFERENCE_CHECKOUT     # spiral RF gaps
    python tests/golden/make_golden.py --injection --ref REFERENCE_CHECKOUT  # central-line injection point
    python tests/golden/make_golden.py --bucket --ref REFERENCE_CHECKOUT     # RF-bucket-matched distribution

The reference imports mpi4py, pyfftw and matplotlib, which are not
installed; tests/golden/shims/ provides single-rank / numpy.fft / no-op
stand-ins (so the space-charge transforms here are numpy's complex64 FFT,
not FFTW).  The fixtures store every input (lattice JSON, z-Taylor stacks,
RF file text, closed-orbit tables, particle matrices) next to the
reference's outputs, so the tests need neither the reference nor this
script.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from pyffa_b200 import synthetic  # noqa: E402

# Coarse map band around the 300 MeV closed orbit so the fixture stays small:
# r 8.0..8.5 m in 5 mm steps, theta step 0.1 deg
GOLD_R = (8.0, 8.5, 0.005)
GOLD_THETA_DEG = 0.1
MAX_ORDER = 2


def build_inputs(tmp):
    bmap_dir = os.path.join(tmp, "bmap")
    cfg_path = synthetic.write_bmap_folder(bmap_dir, MAX_ORDER, r_range=GOLD_R, theta_step_deg=GOLD_THETA_DEG)
    emap_path = synthetic.emap_file(os.path.join(tmp, "emap.txt"), gap_azimuth_deg=(1.0, 4.0),
                                    rf_shift_deg=(0.0, 10.0), voltage=100e3, gap_width=0.2,
                                    E_range=(7.9, 8.6), acc_phi_deg=30.0, ramp_turns=20, npts=201)
    return cfg_path, emap_path


def ref_objects(cfg_path, emap_path, aperture, enable_rf=True):
    from FFAG_ParasAndConversion import FFAG_GlobalParameters
    from FFAG_Field import FFAG_Bfield_analytical, FFAG_EField_new, FFAG_BField_Error
    gp = FFAG_GlobalParameters()
    gp.AddBMap(FFAG_Bfield_analytical(cfg_path, MAX_ORDER))
    gp.AddEMap(FFAG_EField_new(emap_path, enable_rf))
    gp.AddBHarmonics(FFAG_BField_Error([], False))
    if aperture is not None:
        gp.AddAperture(*aperture)
    return gp


def p_bunch(n, seed, inj_spread_ns=0.0, dt=None):
    a = synthetic.centred_bunch(n, seed=seed, sig_x=4e-3, sig_xp=2e-3, sig_z=3e-3, sig_zp=2e-3, sig_delta=2e-3)
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    if inj_spread_ns > 0:
        a[:, 6] = np.sort(rng.uniform(0.0, inj_spread_ns, n))
    return a


def main(ref):
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    import FFAG_track
    from FFAG_Bunch import FFAG_Bunch
    from FFAG_dump import Dumps
    from FFAG_MathTools import RK4_Post_Step_njit
    from FFAG_ParasAndConversion import FFAG_ConversionTools

    conv = FFAG_ConversionTools()
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        cfg_path, emap_path = build_inputs(tmp)
        with open(cfg_path) as f:
            cfg_text = f.read()
        with open(emap_path) as f:
            emap_text = f.read()
        stacks = {}
        for comp in ("Bz", "Bfi", "Br"):
            stacks[comp] = np.stack([np.load(os.path.join(os.path.dirname(cfg_path), f"{comp}_order_{n}.npz"))
                                     [f"{comp}_Taylor_coeff"] for n in range(MAX_ORDER + 1)])
        aperture = (8.02, 8.48, -0.006, 0.006)
        dt = synthetic.design_dt(300.0, 720)
        t0 = 1.0e-9

        # ---- A: single Boris_solve step (all injected; a few outside the aperture; a few not injected)
        gp = ref_objects(cfg_path, emap_path, aperture)
        pa = p_bunch(64, seed=11)
        pa[:4, 0] = [7.99, 8.015, 8.485, 8.51]             # outside the aperture / map edge
        pa[4:8, 4] = np.deg2rad([0.95, 1.0, 1.05, 4.0])    # inside the RF gaps
        va = conv.ConvertPrzek2Vrzek_boris(pa)
        va[:, 9] = 0.3
        va[:, 7] = 1.0
        va[:, 8] = 1.0
        va[60:, 7] = 0.0
        va[60:, 8] = 0.0
        va[8:12, 10:13] = [[1e4, -2e4, 3e3]] * 4            # space-charge field columns
        bunch = FFAG_Bunch(va.copy(), BunchType="Boris")
        rk = FFAG_track.FFAG_RungeKutta()
        m = bunch.LocalBunch
        m_in = m.copy()
        rk.Boris_solve(t0, m, dt,
                       bunch.Malloc_x_cart, bunch.Malloc_y_cart, bunch.Malloc_z_cart,
                       bunch.Malloc_vx_cart, bunch.Malloc_vy_cart, bunch.Malloc_vz_cart,
                       bunch.Malloc_Ex_cart, bunch.Malloc_Ey_cart, bunch.Malloc_Ez_cart,
                       bunch.Malloc_Bx_cart, bunch.Malloc_By_cart, bunch.Malloc_Bz_cart,
                       bunch.Malloc_RF_phase, bunch.Malloc_mod_fi,
                       bunch.Malloc_Bz_interp, bunch.Malloc_Br_interp, bunch.Malloc_Bf_interp,
                       bunch.Malloc_Ez_interp, bunch.Malloc_Er_interp, bunch.Malloc_Ef_interp,
                       bunch.Step_SurviveFlag, bunch.Malloc_RF_shift,
                       bunch.SurvivedNum_Local, bunch.LostNum_Local, gp)
        out["boris1_in"] = m_in
        out["boris1_out"] = m.copy()
        out["boris1_t"] = np.array([t0, dt])

        # ---- B: single RK4 step
        vr = conv.ConvertPrzek2Vrzek(pa)
        vr[:, 9] = 0.3
        vr[:, 7] = 1.0
        vr[:, 8] = 1.0
        vr[60:, 7] = 0.0
        vr[60:, 8] = 0.0
        vr[8:12, 10:13] = [[1e4, -2e4, 3e3]] * 4
        bunch = FFAG_Bunch(vr.copy(), BunchType="RK4")
        m = bunch.LocalBunch
        m_in = m.copy()
        dr, _, _, _ = rk.rk4_step_malloc(FFAG_track.FunctionForAccelerationBunch_dt, t0, m, dt, gp,
                                         bunch.Malloc_Bz_interp, bunch.Malloc_Br_interp, bunch.Malloc_Bf_interp,
                                         bunch.Malloc_Ez_interp, bunch.Malloc_Er_interp, bunch.Malloc_Ef_interp,
                                         bunch.Malloc_mod_fi, bunch.Malloc_RF_shift, bunch.Malloc_RK_dxdt,
                                         bunch.SurvivedNum_Local, bunch.LostNum_Local)
        RK4_Post_Step_njit(m, dr)
        out["rk41_in"] = m_in
        out["rk41_out"] = m.copy()

        # ---- C: tracking loops with injection spread over the first steps (no SC)
        def loop(solver, nsteps, p, sc=None):
            gp_l = ref_objects(cfg_path, emap_path, aperture)
            v = conv.ConvertPrzek2Vrzek_boris(p) if solver == "Boris" else conv.ConvertPrzek2Vrzek(p)
            v[:, 9] = 0.3
            v[:, 15] = np.arange(v.shape[0])
            grid = (8, 32, 32, 6.0) if sc else (64, 128, 128, 12.0)
            b = FFAG_Bunch(v.copy(), marcosize=sc["marcosize"] if sc else 1, sc_grid_size=grid, BunchType=solver)
            if sc:
                b.SEO_fi_axis, b.SEO_Ek_axis = sc["seo"]["fi_axis"], sc["seo"]["Ek_axis"]
                b.SEO_r_matrix, b.SEO_pr_matrix = sc["seo"]["r"], sc["seo"]["pr"]
                b.SEO_perimeter = sc["seo"]["perimeter"]
            lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9},
                  "time_step": dt, "enable_SC": bool(sc), "SC_type": 1, "SC_step": sc["step"] if sc else 20,
                  "step_dumps": Dumps()}
            v_in = b.LocalBunch.copy()
            t_start = -0.5 * dt
            if solver == "Boris":
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC_boris(None, t_start, b, gp_l, lp)
            else:
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC(FFAG_track.FunctionForAccelerationBunch_dt,
                                                                       t_start, b, gp_l, lp)
            return v_in, b.LocalBunch.copy(), t_start

        pl = p_bunch(64, seed=23, inj_spread_ns=4 * dt * 1e9)
        vin, vout, ts = loop("Boris", 240, pl)
        out["borisloop_in"], out["borisloop_out"], out["borisloop_t"] = vin, vout, np.array([ts, dt, 240])
        vin, vout, ts = loop("RK4", 120, pl)
        out["rk4loop_in"], out["rk4loop_out"], out["rk4loop_t"] = vin, vout, np.array([ts, dt, 120])

        # ---- D: space charge: one update through Build_2_5D_SliceGrid_sbs, and a short loop with SC
        from pyffa_b200 import orbit
        seo = orbit.seo_tables(synthetic.lattice_bmap(), np.linspace(290.0, 310.0, 5), nfi=181)
        seo = {k: seo[k] for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}
        ps = synthetic.centred_bunch(3000, seed=5, kind="kv", a_x=3e-3, a_z=2e-3, sig_t=3e-9, fi0=0.3)
        vs = conv.ConvertPrzek2Vrzek_boris(ps)
        vs[:, 7] = 1.0
        vs[:, 8] = 1.0
        vs[:7, 8] = 0.0  # a few lost particles stay out of the deposit
        b = FFAG_Bunch(vs.copy(), marcosize=1e13 / 3000, sc_grid_size=(8, 32, 32, 6.0), BunchType="Boris")
        b.SEO_fi_axis, b.SEO_Ek_axis, b.SEO_r_matrix = seo["fi_axis"], seo["Ek_axis"], seo["r"]
        b.SEO_pr_matrix, b.SEO_perimeter = seo["pr"] + 0.01, seo["perimeter"]
        b.Step_SurviveFlag[:] = b.LocalBunch[:, 8] != 0
        sc_in = b.LocalBunch.copy()
        import pyfftw
        a_buf = pyfftw.empty_aligned((32, 32), dtype="complex64")
        b_buf = pyfftw.empty_aligned((32, 32), dtype="complex64")
        fwd = pyfftw.FFTW(a_buf, b_buf, axes=(0, 1), direction="FFTW_FORWARD")
        inv = pyfftw.FFTW(b_buf, a_buf, axes=(0, 1), direction="FFTW_BACKWARD")
        res = b.Build_2_5D_SliceGrid_sbs(fwd, inv)
        (rho, phi, ex, ez, xmin, xmax, zmin, zmax, BL, _, _, _, _, _, cx, cr0, _, fi_grid) = res
        out["sc_in"] = sc_in
        out["sc_out"] = b.LocalBunch.copy()
        out["sc_rho"], out["sc_phi"], out["sc_ex"], out["sc_ez"] = rho, phi, ex, ez
        out["sc_box"] = np.array([xmin, xmax, zmin, zmax, BL, fi_grid[0], fi_grid[-1]])
        out["sc_params"] = np.array([8, 32, 32, 6.0, 1e13 / 3000 * 1.60217662e-19])
        out["sc_slice_indices"] = b.Malloc_SC_slice_indices[: int((sc_in[:, 8] != 0).sum())].copy()
        out["seo_pr_offset"] = np.array([0.01])
        for k, v in seo.items():
            out["seo_" + k] = v

        psl = synthetic.centred_bunch(1500, seed=9, kind="kv", a_x=3e-3, a_z=2e-3, sig_t=3e-9, fi0=0.0)
        vin, vout, ts = loop("Boris", 12, psl, sc={"seo": seo, "step": 5, "marcosize": 1e13 / 1500})
        out["scloop_in"], out["scloop_out"], out["scloop_t"] = vin, vout, np.array([ts, dt, 12, 5, 1e13 / 1500])

        out["cfg_json"] = np.frombuffer(cfg_text.encode(), dtype=np.uint8)
        out["emap_text"] = np.frombuffer(emap_text.encode(), dtype=np.uint8)
        for comp in ("Bz", "Bfi", "Br"):
            out[f"stack_{comp}"] = stacks[comp][1:]  # order 0 is never read
        out["aperture"] = np.array(aperture)
    path = os.path.join(HERE, "golden_tracking.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def crossing_main(ref):
    """Azimuth-crossing dumps: the reference's Boris and RK4 loops with
    PositionDumpBunch instances registered, and the files they write
    (golden_crossing.npz)."""
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    import FFAG_track
    from FFAG_Bunch import FFAG_Bunch
    from FFAG_dump import Dumps, PositionDumpBunch
    from FFAG_ParasAndConversion import FFAG_ConversionTools

    conv = FFAG_ConversionTools()
    out = {}
    aperture = (8.02, 8.48, -0.006, 0.006)
    dt = synthetic.design_dt(300.0, 720)
    t_start = -0.5 * dt
    # (solver, steps, [(target deg, start, end)]); the last Boris window ends
    # after the run, so the reference never writes that file
    cases = {
        "xb": ("Boris", 300, [(40.0, t_start, t_start + 280 * dt), (100.3, t_start + 50 * dt, t_start + 290 * dt),
                              (7.0, t_start, t_start + 400 * dt)]),
        "xr": ("RK4", 150, [(20.0, t_start, t_start + 140 * dt)]),
    }
    with tempfile.TemporaryDirectory() as tmp:
        cfg_path, emap_path = build_inputs(tmp)
        for key, (solver, nsteps, windows) in cases.items():
            gp = ref_objects(cfg_path, emap_path, aperture)
            p = p_bunch(64, seed=29, inj_spread_ns=4 * dt * 1e9)
            v = conv.ConvertPrzek2Vrzek_boris(p) if solver == "Boris" else conv.ConvertPrzek2Vrzek(p)
            v[:, 9] = 0.3
            v[:, 15] = np.arange(v.shape[0])
            b = FFAG_Bunch(v.copy(), BunchType=solver)
            dumps = Dumps()
            folders = []
            for k, (deg, t0, t1) in enumerate(windows):
                folders.append(os.path.join(tmp, f"{key}_{k}"))
                dumps.add_dump(PositionDumpBunch(deg, t0, t1, save_folder=folders[-1]))
            lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9},
                  "time_step": dt, "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": dumps}
            out[f"{key}_in"] = b.LocalBunch.copy()
            if solver == "Boris":
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC_boris(None, t_start, b, gp, lp)
            else:
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC(FFAG_track.FunctionForAccelerationBunch_dt,
                                                                       t_start, b, gp, lp)
            out[f"{key}_out"] = b.LocalBunch.copy()
            out[f"{key}_t"] = np.array([t_start, dt, nsteps])
            out[f"{key}_windows"] = np.array(windows, dtype=np.float64)
            for k, folder in enumerate(folders):
                files = sorted(os.listdir(folder))
                assert len(files) <= 1, files
                if files:
                    out[f"{key}_file{k}"] = np.frombuffer(files[0].encode(), dtype=np.uint8)
                    out[f"{key}_dump{k}"] = np.load(os.path.join(folder, files[0]))["particles"]
    path = os.path.join(HERE, "golden_crossing.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def mapgen_main(ref):
    """The reference's z-Taylor map generator (Generate_Bmaps,
    src/FFAG_HighOrder.py:828-911, driven as examples/main_Bmap.py:17-75
    does) on two small lattices: the synthetic one (no spiral) and the same
    with a 35-degree spiral (golden_mapgen.npz)."""
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    from numpy.polynomial import Polynomial
    from FFAG_HighOrder import BmapParams_to_ConvexParams, Generate_Bmaps, calculate_s

    out = {}
    for key, spiral in (("flat", 0.0), ("spiral", 35.0)):
        cfg = synthetic.lattice_bmap(r_range=(8.0, 8.5, 0.05), theta_step_deg=0.1)
        B = cfg["Bmap"]
        B["SpiralAngle_deg"] = spiral
        rmin, rmax, rstep = B["rmin_max_step_m"]
        n_r = int((rmax - rmin) / rstep) + 1
        n_fi = int((np.pi * 2 / B["NSector"] - 0.0) / B["theta_step_rad"]) + 1
        fi = np.linspace(0, np.pi * 2 / B["NSector"], n_fi)
        r = np.linspace(rmin, rmax, n_r)
        s = calculate_s(r, 0.0, spiral)
        sfit = Polynomial.fit(r, s, 5)
        Br, Bz, Bfi = Generate_Bmaps(2, r, fi, BmapParams_to_ConvexParams(B), sfit, B["coefficients_tupel"])
        out[f"{key}_cfg"] = np.frombuffer(json.dumps(cfg).encode(), dtype=np.uint8)
        out[f"{key}_Br"], out[f"{key}_Bz"], out[f"{key}_Bfi"] = np.stack(Br), np.stack(Bz), np.stack(Bfi)
    path = os.path.join(HERE, "golden_mapgen.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def seo_main(ref):
    """The reference's closed-orbit search (FFAG_SearchSEO.SearchSEOsControllerVect,
    src/FFAG_track.py:1380-1512, driven as examples/main_SEO.py:13-31) on the
    synthetic lattice (two energies) and on the same lattice with a
    25-degree spiral (two energies), then FFAG_BetaFuncCalc.CalcBetaFunc as
    main_SEO does; the files they write (golden_seo.npz)."""
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    from FFAG_Field import FFAG_Bfield_analytical, FFAG_BField_Error
    from FFAG_ParasAndConversion import FFAG_GlobalParameters
    from FFAG_track import FFAG_SearchSEO
    from FFAG_BetaFunc import FFAG_BetaFuncCalc

    out = {}
    for key, spiral, energies in (("flat", 0.0, [300.0, 330.0]), ("spiral", 25.0, [310.0, 320.0])):
        with tempfile.TemporaryDirectory() as tmp:
            cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
            cfg["Bmap"]["SpiralAngle_deg"] = spiral
            cfg["config"]["folder"] = tmp
            path = os.path.join(tmp, "config_Bmap.json")
            with open(path, "w") as f:
                json.dump(cfg, f)
            FFAG_Bfield_analytical(path, 0, AddNumricalMap=False).UpdataConfig()
            # CalcBetaFunc opens the map folder's order-0 tables (it evaluates
            # the analytic field, so their values are not used)
            shape = (len(np.linspace(7.5, 9.5, 201)), int((np.pi * 2 / 12) / np.deg2rad(0.05)) + 1)
            for comp in ("Br", "Bz", "Bfi"):
                np.savez(os.path.join(tmp, f"{comp}_order_0.npz"), **{f"{comp}_Taylor_coeff": np.zeros(shape)})
            gp = FFAG_GlobalParameters()
            gp.AddBMap(FFAG_Bfield_analytical(path, 0, AddNumricalMap=False))
            gp.AddBHarmonics(FFAG_BField_Error([], False))
            gp.SEO_SaveFold = "seo"
            fold = FFAG_SearchSEO(gp).SearchSEOsControllerVect(np.array(energies))
            with open(path) as f:
                out[f"{key}_cfg"] = np.frombuffer(f.read().encode(), dtype=np.uint8)
            with open(os.path.join(fold, "SEO_ini.txt")) as f:
                text = f.read()
            # the first line names the temporary map folder: keep the rest
            out[f"{key}_ini"] = np.frombuffer(text.split("\n", 1)[1].encode(), dtype=np.uint8)
            out[f"{key}_r"] = np.loadtxt(os.path.join(fold, "SEO_r.txt"), skiprows=1)
            out[f"{key}_pr"] = np.loadtxt(os.path.join(fold, "SEO_pr.txt"), skiprows=1)
            out[f"{key}_Ek"] = np.array(energies)
            # Twiss tables (FFAG_BetaFuncCalc.CalcBetaFunc, src/FFAG_BetaFunc.py:45-240)
            FFAG_BetaFuncCalc().CalcBetaFunc(fold, np.array(energies))
            for name in ("BetaFuncR", "BetaFuncZ", "AlphaFuncR", "AlphaFuncZ", "Bz", "Br", "Bf"):
                out[f"{key}_{name}"] = np.loadtxt(os.path.join(fold, name + ".txt"), skiprows=1)
    path = os.path.join(HERE, "golden_seo.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def bunch_main(ref):
    """The reference's bunch generator (GenerateBunches,
    src/FFAG_Distribution.py:1542-1741) on SEO and Twiss tables it computed
    for the synthetic lattice, with Python's and NumPy's global random
    streams seeded; plus its deterministic helpers (injection point on the
    closed orbit, Twiss at injection).  golden_bunch.npz."""
    import random
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    from FFAG_BetaFunc import FFAG_BetaFuncCalc
    from FFAG_Distribution import GenerateBunches, GetInitRAndFiForInjection, LoadSEOBetaFunc
    from FFAG_Field import FFAG_Bfield_analytical, FFAG_BField_Error
    from FFAG_ParasAndConversion import FFAG_GlobalParameters
    from FFAG_track import FFAG_SearchSEO

    out = {}
    energies = [290.0, 300.0, 310.0, 320.0]
    with tempfile.TemporaryDirectory() as tmp:
        cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
        cfg["config"]["folder"] = tmp
        path = os.path.join(tmp, "config_Bmap.json")
        with open(path, "w") as f:
            json.dump(cfg, f)
        FFAG_Bfield_analytical(path, 0, AddNumricalMap=False).UpdataConfig()
        shape = (201, int((np.pi * 2 / 12) / np.deg2rad(0.05)) + 1)
        for comp in ("Br", "Bz", "Bfi"):
            np.savez(os.path.join(tmp, f"{comp}_order_0.npz"), **{f"{comp}_Taylor_coeff": np.zeros(shape)})
        gp = FFAG_GlobalParameters()
        gp.AddBMap(FFAG_Bfield_analytical(path, 0, AddNumricalMap=False))
        gp.AddBHarmonics(FFAG_BField_Error([], False))
        gp.SEO_SaveFold = "seo"
        fold = FFAG_SearchSEO(gp).SearchSEOsControllerVect(np.array(energies))
        FFAG_BetaFuncCalc().CalcBetaFunc(fold, np.array(energies))
        for name in ("SEO_ini", "SEO_r", "SEO_pr", "BetaFuncR", "BetaFuncZ", "AlphaFuncR", "AlphaFuncZ"):
            with open(os.path.join(fold, name + ".txt")) as f:
                out[f"file_{name}"] = np.frombuffer(f.read().encode(), dtype=np.uint8)
        emap = synthetic.emap_file(os.path.join(tmp, "emap.txt"))
        with open(emap) as f:
            out["file_emap"] = np.frombuffer(f.read().encode(), dtype=np.uint8)
        curve = os.path.join(tmp, "paint.txt")
        with open(curve, "w") as f:
            f.write("t_ns x px y py\n")
            for t, x, px, y, py in ((0.0, 0.0, 0.0, 0.0, 0.0), (2000.0, 0.004, 0.001, 0.003, -0.001)):
                f.write(f"{t} {x} {px} {y} {py}\n")
        with open(curve) as f:
            out["file_paint"] = np.frombuffer(f.read().encode(), dtype=np.uint8)
        SEO_R = np.loadtxt(os.path.join(fold, "SEO_r.txt"), skiprows=1)
        SEO_Pr = np.loadtxt(os.path.join(fold, "SEO_pr.txt"), skiprows=1)
        out["inj_point"] = np.array(GetInitRAndFiForInjection(SEO_R, SEO_Pr, 7.5, 305.0), dtype=np.float64)
        out["inj_twiss"] = np.array(LoadSEOBetaFunc(fold, 305.0, float(out["inj_point"][0])), dtype=np.float64)
        cases = {
            "paint": dict(TransverseDistType="gauss", LongitudeDistType="UniformGauss", PaintEnable=True,
                          ParticleNum=4000, PaintMaxNum=3, PaintTimeInterval=700.0),
            "kv": dict(TransverseDistType="kv", LongitudeDistType="gauss", PaintEnable=False,
                       ParticleNum=8000, PaintMaxNum=1, PaintTimeInterval=700.0),
        }
        for key, extra in cases.items():
            bp = dict(SEO=fold, BmapPATHName=tmp, InjectEk=305.0, InjPosition=7.5, TransverseREmit=0.3,
                      TransverseZEmit=0.2, LongitudeT=72.0, LongitudeDEk=1.0, InjTimeNanoSec=0,
                      PlotFlag=False, PlotRMS=False, PaintCurve=curve, EmapPATHName=emap, **extra)
            random.seed(7)
            np.random.seed(7)
            out[f"{key}_bunch"] = GenerateBunches(dict(bp))
            bp_store = {k: v for k, v in bp.items() if k not in ("SEO", "BmapPATHName", "PaintCurve", "EmapPATHName")}
            out[f"{key}_para"] = np.frombuffer(json.dumps(bp_store).encode(), dtype=np.uint8)
    path = os.path.join(HERE, "golden_bunch.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


# field-error harmonics of the harmonics fixture: one band covering the whole
# map band, one inside it (band edges crossed by the bunch), one high mode
HARMONICS = [{"m": 1, "amp_Gs": 20.0, "phase_deg": 30.0, "rmin": 8.0, "rmax": 8.5},
             {"m": 3, "amp_Gs": 8.0, "phase_deg": -45.0, "rmin": 8.12, "rmax": 8.3},
             {"m": 12, "amp_Gs": 5.0, "phase_deg": 90.0, "rmin": 8.2, "rmax": 8.6}]


def harmonics_main(ref):
    """Boris and RK4 single steps and tracking loops with field-error
    harmonics enabled (FFAG_BField_Error, added by Boris_solve and the RK4
    field function after the map), on the tracking fixture's lattice."""
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    import FFAG_track
    from FFAG_Bunch import FFAG_Bunch
    from FFAG_dump import Dumps
    from FFAG_Field import FFAG_BField_Error
    from FFAG_MathTools import RK4_Post_Step_njit
    from FFAG_ParasAndConversion import FFAG_ConversionTools

    conv = FFAG_ConversionTools()
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        cfg_path, emap_path = build_inputs(tmp)
        cfg_text, emap_text = open(cfg_path).read(), open(emap_path).read()
        stacks = {}
        for comp in ("Bz", "Bfi", "Br"):
            stacks[comp] = np.stack([np.load(os.path.join(os.path.dirname(cfg_path), f"{comp}_order_{n}.npz"))
                                     [f"{comp}_Taylor_coeff"] for n in range(MAX_ORDER + 1)])
        aperture = (8.02, 8.48, -0.006, 0.006)
        dt = synthetic.design_dt(300.0, 720)
        t0 = 1.0e-9

        def gp_h():
            gp = ref_objects(cfg_path, emap_path, aperture)
            gp.AddBHarmonics(FFAG_BField_Error(HARMONICS, True))
            return gp

        pa = p_bunch(64, seed=31)
        pa[4:8, 4] = np.deg2rad([0.95, 1.0, 1.05, 4.0])    # inside the RF gaps
        pa[8:16, 0] = np.linspace(8.10, 8.32, 8)            # across the inner band's edges
        va = conv.ConvertPrzek2Vrzek_boris(pa)
        va[:, 9] = 0.3
        va[:, 7] = 1.0
        va[:, 8] = 1.0
        bunch = FFAG_Bunch(va.copy(), BunchType="Boris")
        m = bunch.LocalBunch
        m_in = m.copy()
        FFAG_track.FFAG_RungeKutta().Boris_solve(
            t0, m, dt, bunch.Malloc_x_cart, bunch.Malloc_y_cart, bunch.Malloc_z_cart,
            bunch.Malloc_vx_cart, bunch.Malloc_vy_cart, bunch.Malloc_vz_cart,
            bunch.Malloc_Ex_cart, bunch.Malloc_Ey_cart, bunch.Malloc_Ez_cart,
            bunch.Malloc_Bx_cart, bunch.Malloc_By_cart, bunch.Malloc_Bz_cart,
            bunch.Malloc_RF_phase, bunch.Malloc_mod_fi,
            bunch.Malloc_Bz_interp, bunch.Malloc_Br_interp, bunch.Malloc_Bf_interp,
            bunch.Malloc_Ez_interp, bunch.Malloc_Er_interp, bunch.Malloc_Ef_interp,
            bunch.Step_SurviveFlag, bunch.Malloc_RF_shift,
            bunch.SurvivedNum_Local, bunch.LostNum_Local, gp_h())
        out["boris1_in"], out["boris1_out"], out["boris1_t"] = m_in, m.copy(), np.array([t0, dt])

        vr = conv.ConvertPrzek2Vrzek(pa)
        vr[:, 9] = 0.3
        vr[:, 7] = 1.0
        vr[:, 8] = 1.0
        bunch = FFAG_Bunch(vr.copy(), BunchType="RK4")
        m = bunch.LocalBunch
        m_in = m.copy()
        dr, _, _, _ = FFAG_track.FFAG_RungeKutta().rk4_step_malloc(
            FFAG_track.FunctionForAccelerationBunch_dt, t0, m, dt, gp_h(),
            bunch.Malloc_Bz_interp, bunch.Malloc_Br_interp, bunch.Malloc_Bf_interp,
            bunch.Malloc_Ez_interp, bunch.Malloc_Er_interp, bunch.Malloc_Ef_interp,
            bunch.Malloc_mod_fi, bunch.Malloc_RF_shift, bunch.Malloc_RK_dxdt,
            bunch.SurvivedNum_Local, bunch.LostNum_Local)
        RK4_Post_Step_njit(m, dr)
        out["rk41_in"], out["rk41_out"] = m_in, m.copy()

        for solver, nsteps in (("Boris", 240), ("RK4", 120)):
            pl = p_bunch(64, seed=37, inj_spread_ns=4 * dt * 1e9)
            v = conv.ConvertPrzek2Vrzek_boris(pl) if solver == "Boris" else conv.ConvertPrzek2Vrzek(pl)
            v[:, 9] = 0.3
            v[:, 15] = np.arange(v.shape[0])
            b = FFAG_Bunch(v.copy(), BunchType=solver)
            lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
                  "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
            v_in = b.LocalBunch.copy()
            ts = -0.5 * dt
            if solver == "Boris":
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC_boris(None, ts, b, gp_h(), lp)
            else:
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC(FFAG_track.FunctionForAccelerationBunch_dt,
                                                                       ts, b, gp_h(), lp)
            key = "borisloop" if solver == "Boris" else "rk4loop"
            out[key + "_in"], out[key + "_out"], out[key + "_t"] = v_in, b.LocalBunch.copy(), np.array([ts, dt, nsteps])

        out["harmonics_json"] = np.frombuffer(json.dumps(HARMONICS).encode(), dtype=np.uint8)
        out["cfg_json"] = np.frombuffer(cfg_text.encode(), dtype=np.uint8)
        out["emap_text"] = np.frombuffer(emap_text.encode(), dtype=np.uint8)
        for comp in ("Bz", "Bfi", "Br"):
            out[f"stack_{comp}"] = stacks[comp][1:]
        out["aperture"] = np.array(aperture)
        from pyffa_b200 import orbit
        seo = orbit.seo_tables(synthetic.lattice_bmap(), np.linspace(290.0, 310.0, 5), nfi=181)
        for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter"):
            out["seo_" + k] = seo[k]
    path = os.path.join(HERE, "golden_harmonics.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


# Spiral RF gap of the spiral fixture (synthetic.spiral_emap_folder): two gaps
# whose windows overlap, so the first-gap rule is exercised
SPIRAL = dict(alpha_deg=40.0, r_ref=8.2, r_axis=(7.95, 8.55, 61), pad_deg=1.0, nphi=121, sigma=0.02,
              gap_azimuth_deg=(1.0, 4.0), rf_shift_deg=(0.0, 25.0), voltage=150e3, gap_width=0.2,
              acc_phi_deg=30.0, ramp_turns=20, npts=201)


def spiral_main(ref):
    """Spiral RF gaps (FFAG_EField_spiral): the reference's own field lookup
    (Interpolation2D_EMap) on scattered points, Boris and RK4 single steps
    and tracking loops through the gaps, on the tracking fixture's lattice."""
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    import FFAG_track
    from FFAG_Bunch import FFAG_Bunch
    from FFAG_dump import Dumps
    from FFAG_Field import FFAG_EField_spiral
    from FFAG_MathTools import RK4_Post_Step_njit
    from FFAG_ParasAndConversion import FFAG_ConversionTools

    conv = FFAG_ConversionTools()
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        cfg_path, emap_fixed = build_inputs(tmp)
        sp_dir = os.path.join(tmp, "spiral")
        emap_path = synthetic.spiral_emap_folder(sp_dir, **SPIRAL)
        aperture = (8.02, 8.48, -0.006, 0.006)
        dt = synthetic.design_dt(300.0, 720)
        t0 = 1.0e-9

        def gp_s():
            gp = ref_objects(cfg_path, emap_fixed, aperture)
            gp.AddEMap(FFAG_EField_spiral(emap_path, True))
            return gp

        # ---- the field lookup itself on scattered points
        rng = np.random.Generator(np.random.PCG64(41))
        n = 4000
        r = rng.uniform(7.9, 8.6, n)                        # beyond both ends of the map's r axis too
        fi = np.concatenate([rng.uniform(-4 * np.pi, 4 * np.pi, n // 2),
                             np.deg2rad(rng.uniform(-3.0, 9.0, n // 2)) + 2 * np.pi * rng.integers(-3, 4, n // 2)])
        z = rng.uniform(-0.01, 0.01, n)
        em = FFAG_EField_spiral(emap_path, True)
        Er, Ez, Efi = np.zeros(n), np.zeros(n), np.zeros(n)
        hit = np.zeros(n, dtype=np.int32)
        em.Interpolation2D_EMap(r, fi, z, Er, Ez, Efi, hit, v0_volt=1.3e5)
        out["lookup_in"] = np.stack([r, fi, z], 1)
        out["lookup_out"] = np.stack([Er, Ez, Efi], 1)
        out["lookup_hit"] = hit
        out["lookup_v0"] = np.array([1.3e5])

        # ---- single steps with particles across both gap windows
        pa = p_bunch(64, seed=43)
        pa[:40, 4] = np.deg2rad(np.linspace(-2.0, 7.0, 40))
        pa[40:48, 0] = np.linspace(8.03, 8.47, 8)
        pa[40:48, 4] = np.deg2rad(2.5)
        va = conv.ConvertPrzek2Vrzek_boris(pa)
        va[:, 9] = 0.3
        va[:, 7] = 1.0
        va[:, 8] = 1.0
        va[60:, 7] = 0.0
        va[60:, 8] = 0.0
        bunch = FFAG_Bunch(va.copy(), BunchType="Boris")
        m = bunch.LocalBunch
        m_in = m.copy()
        FFAG_track.FFAG_RungeKutta().Boris_solve(
            t0, m, dt, bunch.Malloc_x_cart, bunch.Malloc_y_cart, bunch.Malloc_z_cart,
            bunch.Malloc_vx_cart, bunch.Malloc_vy_cart, bunch.Malloc_vz_cart,
            bunch.Malloc_Ex_cart, bunch.Malloc_Ey_cart, bunch.Malloc_Ez_cart,
            bunch.Malloc_Bx_cart, bunch.Malloc_By_cart, bunch.Malloc_Bz_cart,
            bunch.Malloc_RF_phase, bunch.Malloc_mod_fi,
            bunch.Malloc_Bz_interp, bunch.Malloc_Br_interp, bunch.Malloc_Bf_interp,
            bunch.Malloc_Ez_interp, bunch.Malloc_Er_interp, bunch.Malloc_Ef_interp,
            bunch.Step_SurviveFlag, bunch.Malloc_RF_shift,
            bunch.SurvivedNum_Local, bunch.LostNum_Local, gp_s())
        out["boris1_in"], out["boris1_out"], out["boris1_t"] = m_in, m.copy(), np.array([t0, dt])

        vr = conv.ConvertPrzek2Vrzek(pa)
        vr[:, 9] = 0.3
        vr[:, 7] = 1.0
        vr[:, 8] = 1.0
        vr[60:, 7] = 0.0
        vr[60:, 8] = 0.0
        bunch = FFAG_Bunch(vr.copy(), BunchType="RK4")
        m = bunch.LocalBunch
        m_in = m.copy()
        dr, _, _, _ = FFAG_track.FFAG_RungeKutta().rk4_step_malloc(
            FFAG_track.FunctionForAccelerationBunch_dt, t0, m, dt, gp_s(),
            bunch.Malloc_Bz_interp, bunch.Malloc_Br_interp, bunch.Malloc_Bf_interp,
            bunch.Malloc_Ez_interp, bunch.Malloc_Er_interp, bunch.Malloc_Ef_interp,
            bunch.Malloc_mod_fi, bunch.Malloc_RF_shift, bunch.Malloc_RK_dxdt,
            bunch.SurvivedNum_Local, bunch.LostNum_Local)
        RK4_Post_Step_njit(m, dr)
        out["rk41_in"], out["rk41_out"] = m_in, m.copy()

        # ---- loops that carry the bunch through both gaps
        for solver, nsteps in (("Boris", 240), ("RK4", 120)):
            pl = p_bunch(64, seed=47, inj_spread_ns=4 * dt * 1e9)
            pl[:, 4] = np.deg2rad(rng.uniform(-4.0, 0.0, 64))
            v = conv.ConvertPrzek2Vrzek_boris(pl) if solver == "Boris" else conv.ConvertPrzek2Vrzek(pl)
            v[:, 9] = 0.3
            v[:, 15] = np.arange(v.shape[0])
            b = FFAG_Bunch(v.copy(), BunchType=solver)
            lp = {"stop_condition": {"max_stepsN": nsteps, "max_turn": 1e9, "max_time": 1e9}, "time_step": dt,
                  "enable_SC": False, "SC_type": 1, "SC_step": 20, "step_dumps": Dumps()}
            v_in = b.LocalBunch.copy()
            ts = -0.5 * dt
            if solver == "Boris":
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC_boris(None, ts, b, gp_s(), lp)
            else:
                FFAG_track.FFAG_RungeKutta().rk4_solve_dt_bunch3_withSC(FFAG_track.FunctionForAccelerationBunch_dt,
                                                                       ts, b, gp_s(), lp)
            key = "borisloop" if solver == "Boris" else "rk4loop"
            out[key + "_in"], out[key + "_out"], out[key + "_t"] = v_in, b.LocalBunch.copy(), np.array([ts, dt, nsteps])

        with open(cfg_path) as f:
            out["cfg_json"] = np.frombuffer(f.read().encode(), dtype=np.uint8)
        for name in ("emap.txt", "Er_coef.txt", "Ez_coef.txt", "Ephi_coef.txt"):
            with open(os.path.join(sp_dir, name)) as f:
                out["file_" + name.replace(".txt", "")] = np.frombuffer(f.read().encode(), dtype=np.uint8)
        stacks = {}
        for comp in ("Bz", "Bfi", "Br"):
            stacks[comp] = np.stack([np.load(os.path.join(os.path.dirname(cfg_path), f"{comp}_order_{n}.npz"))
                                     [f"{comp}_Taylor_coeff"] for n in range(MAX_ORDER + 1)])
            out[f"stack_{comp}"] = stacks[comp][1:]
        out["aperture"] = np.array(aperture)
        out["spiral_json"] = np.frombuffer(json.dumps(SPIRAL).encode(), dtype=np.uint8)
    path = os.path.join(HERE, "golden_spiral.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def injection_main(ref):
    """The injection point on the closed orbit where an injection central line
    crosses it (GetInitRAndFiForInjection, src/FFAG_Distribution.py:1347-1414,
    central-line branch).  The reference's function raises at its last line
    (it indexes the scalar azimuth, `theta_rad[0]`), so the fixture runs the
    same steps through the reference's own helpers -- My1p5DInterp,
    CentralLine2Segments, FindIntersectionVect, xy2rfi_m2p180 -- and stores
    what the function computes before that line; it also records that the
    function itself raises."""
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    from FFAG_Distribution import GetInitRAndFiForInjection
    from FFAG_MathTools import FFAG_interpolation
    from FFAG_ParasAndConversion import FFAG_ConversionTools
    from FFAG_Utils import FFAG_GeometryCalc, FFAG_SegmentTools
    from pyffa_b200 import orbit
    tab = orbit.seo_tables(synthetic.lattice_bmap(), np.linspace(290.0, 310.0, 5), nfi=361)
    fi, Ek_axis = tab["fi_axis"], tab["Ek_axis"]
    SEO_R = np.zeros((len(Ek_axis) + 1, len(fi) + 1))
    SEO_R[0, 1:], SEO_R[1:, 0], SEO_R[1:, 1:] = fi, Ek_axis, tab["r"]
    SEO_Pr = SEO_R.copy()
    SEO_Pr[1:, 1:] = tab["pr"]
    rng = np.random.Generator(np.random.PCG64(53))
    lines, cases = [], []
    for k in range(8):
        a = np.deg2rad(rng.uniform(0.0, 360.0))
        tilt = np.deg2rad(rng.uniform(-20.0, 20.0))
        rr = np.linspace(7.6, 8.9, 5 + k)
        bend = 0.002 * rng.standard_normal(len(rr))
        ang = a + np.tan(tilt) * (rr - 8.2) / 8.2 + bend
        lines.append(np.column_stack([rr * np.cos(ang), rr * np.sin(ang)]))
    out = {}
    raised = 0
    for k, CL in enumerate(lines):
        Ek = float(rng.uniform(291.0, 309.0))
        try:
            GetInitRAndFiForInjection(SEO_R, SEO_Pr, CL, Ek)
        except IndexError:
            raised += 1
        R, P = SEO_R[1:, 1:], SEO_Pr[1:, 1:]
        r_fi, _ = FFAG_interpolation().My1p5DInterp(Ek_axis, R)(np.array([Ek]))
        pr_fi, _ = FFAG_interpolation().My1p5DInterp(Ek_axis, P)(np.array([Ek]))
        traj = np.column_stack((r_fi[0] * np.cos(fi), r_fi[0] * np.sin(fi)))
        traj = np.vstack((traj, traj[1, :]))
        seo_seg = FFAG_SegmentTools().CentralLine2Segments(traj)
        cl_seg = FFAG_SegmentTools().CentralLine2Segments(CL)
        flag, dA1, dA2, _, _ = FFAG_GeometryCalc().FindIntersectionVect(seo_seg, cl_seg)
        ii, jj = np.where(flag)
        i, j = ii[0], jj[0]
        pre, post = abs(dA1[i, j]), abs(dA2[i, j])
        tot = pre + post
        point = (pre - tot) / (0 - tot) * seo_seg[i, 0:2] + (pre - 0) / (tot - 0) * seo_seg[i, 2:4]
        th, r, _ = FFAG_ConversionTools().xy2rfi_m2p180(point[0], point[1])
        cases.append([Ek, float(th), float(r), float(pr_fi[0, i]), float(i), float(j)])
        out[f"line_{k}"] = CL
    out["cases"] = np.array(cases)
    out["seo_r"], out["seo_pr"] = SEO_R, SEO_Pr
    out["reference_raised"] = np.array([raised])
    path = os.path.join(HERE, "golden_injection.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes; the reference raised on", raised, "of", len(lines))


def bucket_main(ref):
    """The RF bucket of the 'match' longitudinal distribution (FFAG_bucket,
    src/FFAG_bucket.py) with the generator's parameters (step 20 ns, 18000
    steps) on a closed-orbit frequency table of the synthetic lattice: its
    starting points, stability flags, box limits, H on the grid, the
    centre-line H-span relation, thresholds for three bunch lengths and one
    sample of its (unseeded) rejection draw."""
    sys.path.insert(0, os.path.join(HERE, "shims"))
    sys.path.insert(0, os.path.join(ref, "src"))
    from FFAG_bucket import FFAG_bucket
    from FFAG_MathTools import FFAG_interpolation
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "resultsSEO"))
        Ek = np.linspace(250.0, 350.0, 21)
        f = 1.0 / synthetic.revolution_time(Ek)
        rows = np.column_stack([np.arange(len(Ek)), Ek, synthetic.orbit_radius(Ek), np.zeros(len(Ek)), f])
        path = os.path.join(tmp, "resultsSEO", "SEO_ini.txt")
        with open(path, "w") as fh:
            fh.write("synthetic closed-orbit table\nidx Ek r pr f\n")
            np.savetxt(fh, rows, fmt="%.17e")
        out["seo_ini_text"] = np.frombuffer(open(path).read().encode(), dtype=np.uint8)
        for k, (fi0, U0) in enumerate(((30.0, 100e3), (20.0, 150e3))):
            b = FFAG_bucket(tmp, Ek0=300.0, fi0=fi0, U0=U0, step_t=20e-9, step_N=18000)
            b.build_H()
            H, L = b.compute_center_H_vs_span()
            thr = []
            for Lt in (30.0, 80.0, 1e4):
                Lu = float(np.clip(Lt, L.min(), L.max()))
                o = np.argsort(L)
                thr.append(float(FFAG_interpolation().linear_interpolation(L[o], H[o])(Lu)))
            t_ns, Ek_s, H_thr = b.scatter_filter_by_span(20000, 80.0, show=False)
            assert abs(H_thr - thr[1]) == 0.0
            out[f"b{k}_params"] = np.array([fi0, U0, b.G.Tc, b.G.w0, b.zd_u])
            out[f"b{k}_X_in"] = b.X_in
            out[f"b{k}_stable"] = np.stack([b.stable_fwd, b.stable_rev])
            out[f"b{k}_limits"] = np.array([b.x_min_plot, b.x_max_plot, b.y_min_plot, b.y_max_plot,
                                            b.x_min_sample, b.x_max_sample, b.y_min_sample, b.y_max_sample])
            out[f"b{k}_tr_end"] = np.stack([b.tr_fwd[-1], b.tr_rev[-1]])
            out[f"b{k}_H"] = np.stack([b.q_grid, b.p_grid, b.Hq_rel, b.Hp_rel])
            out[f"b{k}_H0"] = np.array([b.H00, b.H_sep])
            out[f"b{k}_HL"] = np.stack([H, L])
            out[f"b{k}_thr"] = np.array(thr)
            out[f"b{k}_sample"] = np.stack([t_ns, Ek_s], 1)
    path = os.path.join(HERE, "golden_bucket.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description="Generate golden vectors by running the reference's own code.")
    ap.add_argument("--ref", default=os.environ.get("PYFFA_REFERENCE"),
                    help="checkout of the reference project (or set PYFFA_REFERENCE)")
    kind = ap.add_mutually_exclusive_group()
    for k in ("bunch", "seo", "mapgen", "crossing", "harmonics", "spiral", "injection", "bucket"):
        kind.add_argument("--" + k, action="store_true")
    args = ap.parse_args()
    if not args.ref:
        ap.error("the reference checkout is required: --ref PATH or PYFFA_REFERENCE=PATH")
    if args.bucket:
        bucket_main(args.ref)
    elif args.injection:
        injection_main(args.ref)
    elif args.spiral:
        spiral_main(args.ref)
    elif args.harmonics:
        harmonics_main(args.ref)
    elif args.bunch:
        bunch_main(args.ref)
    elif args.seo:
        seo_main(args.ref)
    elif args.mapgen:
        mapgen_main(args.ref)
    elif args.crossing:
        crossing_main(args.ref)
    else:
        main(args.ref)
