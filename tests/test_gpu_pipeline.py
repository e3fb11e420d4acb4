"""The reference's whole workflow on the GPU path, end to end:
main_Bmap (z-Taylor tables) -> main_SEO (closed orbits, Twiss) ->
main_track (generated, painted bunch; Boris loop with all four dump kinds) ->
main_track -r (restart from the step dump), which must continue the first
run: the restarted bunch at the end equals the uninterrupted one."""
import json
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _write(path, obj):
    with open(path, "w") as f:
        json.dump(obj, f, indent=1)
    return path


@pytest.fixture(scope="module")
def workdir():
    from pyffa_b200 import mapgen, seo, synthetic
    d = tempfile.mkdtemp()
    mapdir = os.path.join(d, "bmap")
    os.makedirs(mapdir)
    cfg = synthetic.lattice_bmap(r_range=(7.5, 9.5, 0.01), theta_step_deg=0.05)
    cfg["config"] = {"folder": ".", "expand_order": 2}
    mapgen.main_Bmap(_write(os.path.join(mapdir, "config_Bmap.json"), cfg))
    seo_cfg = {"config": {"start_Ek": 290.0, "end_Ek": 320.0, "delta_Ek": 10.0, "extra_Ek": [],
                          "Bmap_path": mapdir, "SEO_folder": "seo"},
               "BHarmonics": {"enable": False, "harmonics": []}}
    seo.main_SEO(_write(os.path.join(d, "config_SEO.json"), seo_cfg))
    emap = synthetic.emap_file(os.path.join(d, "emap.txt"))
    with open(os.path.join(d, "paint.txt"), "w") as f:
        f.write("t_ns x px y py\n0 0 0 0 0\n250 0.003 0.001 0.002 0.0\n")
    T = 1 / np.loadtxt(os.path.join(mapdir, "seo", "SEO_ini.txt"), skiprows=2)[1, 4]
    out = os.path.join(d, "out")
    track = {
        "BmapAndSEO": {"maps": mapdir, "max_order": 2, "SEO_FileName": "seo"},
        "Emap": {"maps": emap, "enable": True},
        "track": {"start_EkMeV": 305.0, "start_azimuth": 0.0, "time_step": T / 720, "solver_type": 1,
                  "stop_condition": {"max_stepsN": 2500, "max_turn": 1e9, "max_time": 1.0}},
        "SC": {"enable_SC": False, "SC_type": 1, "grid_size_rfz": [8, 32, 32, 6.0], "step": 20},
        "BunchPara": {"ParticleDensity": 1e8, "ParticleNum": 300, "TransverseREmit": 0.3, "TransverseZEmit": 0.3,
                      "LongitudeT": 20.0, "LongitudeDEk": 0.5, "InjTimeNanoSec": 0,
                      "TransverseDistType": "gauss", "LongitudeDistType": "UniformGauss", "Seed": 3},
        "Paint": {"enable": True, "MaxBunchNum": 2, "TimeInterval": 100.0, "Curve": os.path.join(d, "paint.txt")},
        "Aperture": {"enable": True, "Rmin": 7.6, "Rmax": 9.4, "Zmin": -0.05, "Zmax": 0.05},
        "check": {"CheckBunch": False, "PlotRMS": False},
        "DumpPara": {"modules": [
            {"type": "StepDumpBunch", "start_time": 300e-9, "end_time": 350e-9, "interval_time": 100e-9,
             "save_folder": os.path.join(out, "restart"), "filtter_survive_paticles": True},
            {"type": "PositionDumpBunch", "start_time": 0.0, "end_time": 600e-9, "dump_azimuth": [180.0],
             "save_folder": os.path.join(out, "xing")},
            {"type": "StepDump", "start_time": 0.0, "end_time": 600e-9, "interval_time": 100e-9,
             "tracked_particle_id_global": [0, 5, 17], "save_folder": os.path.join(out, "step")},
            {"type": "PositionDump", "start_time": 0.0, "end_time": 600e-9, "dump_azimuth": [90.0],
             "num_particles_to_dump_global": [1, 2, 3], "save_folder": os.path.join(out, "pos")},
        ]},
    }
    return {"dir": d, "mapdir": mapdir, "track": track, "out": out}


def test_pipeline_and_restart(workdir):
    from pyffa_b200 import main_track
    cfg = workdir["track"]
    path = _write(os.path.join(workdir["dir"], "config_track.json"), cfg)
    a = main_track.main(path, verbose=False).LocalBunch
    assert a.shape == (600, 16)
    assert (a[:, 7] == 1).all() and (a[:, 8] == 1).sum() > 500

    out = workdir["out"]
    files = os.listdir(os.path.join(out, "restart"))
    assert len(files) == 1 and files[0].startswith("time_")
    assert os.listdir(os.path.join(out, "xing")) == ["crossing_angle_180.0_start_0.000_end_600.000_rank_0.npz"]
    x = np.load(os.path.join(out, "xing", os.listdir(os.path.join(out, "xing"))[0]))["particles"]
    assert x.shape[1] == 17 and x.shape[0] >= 500
    assert np.all(np.abs(np.mod(x[:, 4], 2 * np.pi) - np.pi) < 0.05)
    step_files = sorted(os.listdir(os.path.join(out, "step")))
    assert step_files == sorted(f"particle_{g}_rank_0.npz" for g in (0, 5, 17))
    s = np.load(os.path.join(out, "step", "particle_5_rank_0.npz"))["particles"]
    assert s.shape[1] == 17 and s.shape[0] >= 5 and np.all(np.diff(s[:, 16]) > 0)
    pos_files = sorted(os.listdir(os.path.join(out, "pos")))
    assert pos_files == sorted(f"particle_{g}_angle_90.0_rank_0.npz" for g in (1, 2, 3))

    # restart from the step dump and run the remaining steps
    rfile = os.path.join(out, "restart", files[0])
    t_dump = np.load(rfile)["particles"][0, -1]
    # the driver starts at -200.0 * 1e-9 (examples/main_track.py:266) and adds dt step by step
    ext = np.add.accumulate(np.concatenate([[-200.0 * 1e-9], np.full(3000, cfg["track"]["time_step"])]))
    k = int(np.nonzero(ext == t_dump)[0][0])
    cfg2 = json.loads(json.dumps(cfg))
    cfg2["DumpPara"]["modules"] = []
    cfg2["track"]["stop_condition"]["max_stepsN"] = 2500 - k
    path2 = _write(os.path.join(workdir["dir"], "config_restart.json"), cfg2)
    b = main_track.main(path2, rfile, verbose=False).LocalBunch
    ia = {int(g): i for i, g in enumerate(a[:, 15])}
    rows = np.array([ia[int(g)] for g in b[:, 15]])
    a2 = a[rows]
    assert np.array_equal(a2[:, 8], b[:, 8])
    for c in (0, 4, 5, 9):
        assert np.max(np.abs(b[:, c] - a2[:, c]) / np.abs(a2[:, c])) <= 1e-9, c
    for c in (1, 2, 3):
        assert np.max(np.abs(b[:, c] - a2[:, c])) <= 1e-7 * np.abs(a2[:, c]).max(), c
