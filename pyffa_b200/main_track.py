"""The tracking driver: main_track (examples/main_track.py:48-366) on the GPU path.

``main(config_file, restart_bunch=None)`` reads the reference's
config_track.json (keys BmapAndSEO, Emap, track, SC, BunchPara, Paint,
Aperture, DumpPara, check), builds the field, RF, closed-orbit tables and the
bunch (generated, or read back from a restart dump), registers the dumps and
runs the Boris (solver_type 1) or RK4 (solver_type 0) loop of
pyffa_b200.track.  ``Tracker.from_json(path, restart=None).run()`` is the same
as an object.

Differences from the reference driver: the bunch generator is seeded
(``BunchPara.Seed``, default 0); there is no MPI split (one process tracks
the whole bunch; see bunch.divide_variables for the reference's split).
"""
from __future__ import annotations

import json
import os

import numpy as np

from .bunch import FFAG_Bunch
from .constants import COLUMNS, FFAG_ConversionTools, FFAG_GlobalParameters
from .distribution import GenerateBunches
from .dump import Dumps, PositionDump, PositionDumpBunch, StepDump, StepDumpBunch
from .fields import (FFAG_Bfield_analytical, FFAG_BField_Error, FFAG_EField_new, FFAG_EField_spiral,
                     parse_emap_file)
from .seo import LoadSEOParams
from .track import FFAG_RungeKutta


def load_config_from_json(json_path):
    with open(json_path) as f:
        return json.load(f)


def wrap_0_2pi(x):
    return x % (2.0 * np.pi)


def calc_injection_rf_phase(EMap, Azimuth_start, t_start, T0, Ek_inj, gap_idx=0):
    """RF phase of the bunch at t_start such that the gap is crossed at the
    accelerating phase (examples/main_track.py:26-45): the gap azimuth, for
    spiral gaps where the closed orbit of the injection energy meets gap 0,
    shifted by the gap's offset from gap 0."""
    phi_start = wrap_0_2pi(Azimuth_start)
    if EMap.GapType == "fixed":
        phi_gap = EMap.gap_azimuths[gap_idx]
    elif EMap.GapType == "spiral":
        phi_gap = EMap.phi_gap_interp_unwrapped(Ek_inj) + (EMap.gap_azimuths[gap_idx] - EMap.gap_azimuths[0])
    else:
        raise ValueError("EMap.type must be 'fixed' or 'spiral'")
    dphi_orbit = phi_gap - phi_start
    return EMap.acc_phi0 - EMap.harmonic * dphi_orbit - EMap.harmonic * 2.0 * np.pi * (0.0 - t_start) / T0


def build_dumps(config) -> Dumps:
    """DumpPara.modules -> Dumps (examples/main_track.py:165-205)."""
    dumps = Dumps()
    for dc in config.get("DumpPara", {}).get("modules", []):
        t = dc["type"]
        if t == "StepDump":
            dumps.add_dump(StepDump(dc["start_time"], dc["end_time"], dc["interval_time"],
                                    dc["tracked_particle_id_global"], save_folder=dc["save_folder"]))
        elif t == "PositionDump":
            for az in dc["dump_azimuth"]:
                dumps.add_dump(PositionDump(az, dc["start_time"], dc["end_time"], dc["num_particles_to_dump_global"],
                                            save_folder=dc["save_folder"], allow_existing=True))
        elif t == "StepDumpBunch":
            dumps.add_dump(StepDumpBunch(dc["start_time"], dc["end_time"], dc["interval_time"],
                                         save_folder=dc["save_folder"],
                                         filter_survive_flag=dc["filtter_survive_paticles"]))
        elif t == "PositionDumpBunch":
            for az in dc["dump_azimuth"]:
                dumps.add_dump(PositionDumpBunch(az, dc["start_time"], dc["end_time"], save_folder=dc["save_folder"],
                                                 allow_existing=True))
        else:
            raise ValueError(f"unknown dump type {t!r}")
    return dumps


class Tracker:
    """One tracking run of a config_track.json."""

    def __init__(self, config: dict, restart=None, precision="fp64", verbose=True, device=None):
        self.config = config
        self.restart = restart
        self.precision = precision
        self.verbose = verbose
        self.device = device
        self.bunch = None

    @classmethod
    def from_json(cls, path, restart=None, **kw):
        return cls(load_config_from_json(path), restart, **kw)

    def _initial_bunch(self, BunchPara):
        conv = FFAG_ConversionTools()
        if self.restart is not None:
            if not os.path.exists(self.restart):
                raise FileNotFoundError(f"Error: restart_bunch file '{self.restart}' not found.")
            if self.restart.endswith(".npz"):
                p = np.load(self.restart)["particles"]
            else:
                p = np.loadtxt(self.restart, delimiter=",")
            p = p[np.argsort(p[:, COLUMNS["inj_t"]], kind="stable")]
            return p, conv.ConvertPrzek2Vrzek(p), conv.ConvertPrzek2Vrzek_boris(p)
        p = GenerateBunches(BunchPara)
        p = p[np.argsort(p[:, COLUMNS["inj_t"]], kind="stable")]
        v, vb = conv.ConvertPrzek2Vrzek(p), conv.ConvertPrzek2Vrzek_boris(p)
        v[:, COLUMNS["Global_ID"]] = np.arange(p.shape[0])
        vb[:, COLUMNS["Global_ID"]] = np.arange(p.shape[0])
        return p, v, vb

    def run(self):
        cfg = self.config
        bmap_dir = cfg["BmapAndSEO"]["maps"]
        max_order = cfg["BmapAndSEO"]["max_order"]
        seo_dir = os.path.join(bmap_dir, cfg["BmapAndSEO"]["SEO_FileName"])
        emap_path = cfg["Emap"]["maps"]
        Ek = cfg["track"]["start_EkMeV"]
        az0 = cfg["track"]["start_azimuth"]
        BunchPara = dict(cfg["BunchPara"])
        paint = cfg["Paint"]
        BunchPara.update(PlotFlag=cfg.get("check", {}).get("CheckBunch", False),
                         PlotRMS=cfg.get("check", {}).get("PlotRMS", False), BmapPATHName=bmap_dir, SEO=seo_dir,
                         InjectEk=Ek, InjPosition=az0, PaintEnable=paint["enable"], PaintMaxNum=paint["MaxBunchNum"],
                         PaintTimeInterval=paint["TimeInterval"], PaintCurve=paint["Curve"],
                         EmapPATHName=emap_path)
        BunchPara.setdefault("Seed", 0)
        p, v, vb = self._initial_bunch(BunchPara)
        dumps = build_dumps(cfg)

        SEO_inj, bmap_path, SEO_info = LoadSEOParams(os.path.join(seo_dir, "SEO_ini.txt"), Ek)
        r_info = np.loadtxt(os.path.join(seo_dir, "SEO_r.txt"), skiprows=1)
        pr_info = np.loadtxt(os.path.join(seo_dir, "SEO_pr.txt"), skiprows=1)
        gp = FFAG_GlobalParameters()
        gp.AddBMap(FFAG_Bfield_analytical(os.path.join(bmap_path, "config_Bmap.json"), max_order))
        header, _ = parse_emap_file(emap_path)
        gap_type = str(header.get("gap_model", "fixed")).strip().lower()
        if gap_type == "fixed":
            emap = FFAG_EField_new(emap_path, cfg["Emap"]["enable"])
        elif gap_type == "spiral":
            emap = FFAG_EField_spiral(emap_path, cfg["Emap"]["enable"])
        else:
            raise ValueError(f"Unknown Emap gap type: {gap_type!r}")
        gp.AddEMap(emap)
        gp.AddSEOInfo(SEO_info)
        seo_cfg = os.path.join(seo_dir, "config_SEO.json")
        if os.path.exists(seo_cfg):
            h = load_config_from_json(seo_cfg).get("BHarmonics", {"harmonics": [], "enable": False})
            gp.AddBHarmonics(FFAG_BField_Error(h["harmonics"], h["enable"]))
        ap = cfg["Aperture"]
        if ap["enable"]:
            gp.AddAperture(ap["Rmin"], ap["Rmax"], ap["Zmin"], ap["Zmax"])

        t_start = -200.0 * 1e-9
        lp = {"stop_condition": cfg["track"]["stop_condition"], "time_step": cfg["track"]["time_step"],
              "step_dumps": dumps, "enable_SC": cfg["SC"]["enable_SC"], "SC_type": cfg["SC"]["SC_type"],
              "SC_step": cfg["SC"]["step"]}
        grid = tuple(cfg["SC"]["grid_size_rfz"])
        if self.restart is not None:
            t_start = p[0, -1]
        else:
            phase = calc_injection_rf_phase(emap, az0, t_start, SEO_inj[3], SEO_inj[0], gap_idx=0)
            v[:, COLUMNS["RF_phase"]] = phase
            vb[:, COLUMNS["RF_phase"]] = phase
        solver = cfg["track"]["solver_type"]
        if solver not in (0, 1):
            raise ValueError("solver_type must be 0 or 1")
        kind = "Boris" if solver == 1 else "RK4"
        b = FFAG_Bunch(vb if solver == 1 else v, marcosize=BunchPara["ParticleDensity"], sc_grid_size=grid,
                       BunchType=kind, device=self.device)
        b.SEO_fi_axis, b.SEO_Ek_axis = r_info[0, 1:], r_info[1:, 0]
        b.SEO_r_matrix, b.SEO_pr_matrix = r_info[1:, 1:], pr_info[1:, 1:]
        b.SEO_perimeter = SEO_info[:, 8]
        if self.restart is not None:
            b.restore_from_restart_matrix()
        rk = FFAG_RungeKutta(precision=self.precision, verbose=self.verbose)
        if solver == 1:
            rk.rk4_solve_dt_bunch3_withSC_boris(None, t_start, b, gp, lp)
        else:
            rk.rk4_solve_dt_bunch3_withSC(None, t_start, b, gp, lp)
        self.bunch = b
        self.last_run = rk.last_run
        return b


def main(config_file, restart_bunch=None, **kw):
    """examples/main_track.py main()."""
    return Tracker.from_json(config_file, restart_bunch, **kw).run()


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="B200 tracking driver (config_track.json)")
    ap.add_argument("config", nargs="?", default="./config_track.json")
    ap.add_argument("-r", "--restart", default=None)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32c", "fp32"])
    a = ap.parse_args()
    main(a.config, a.restart, precision=a.precision)
