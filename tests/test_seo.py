"""Closed-orbit search and SEO files (FFAG_SearchSEO, src/FFAG_track.py:1142-1621).

tests/golden/golden_seo.npz holds what the reference's
SearchSEOsControllerVect wrote for the synthetic lattice (300 and 330 MeV)
and for the same lattice with a 25-degree spiral (310 and 320 MeV), and
the Twiss tables of FFAG_BetaFuncCalc (tests/golden/make_golden.py --seo).
The search runs on the host rules of pyffa_b200.seo with either the
oracle's azimuth tracker (CPU) or the library's (GPU)."""
import json
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from pyffa_b200 import seo as S
from pyffa_b200.constants import FFAG_GlobalParameters
from pyffa_b200.fields import FFAG_Bfield_analytical

from .fixtures import HERE

GOLDEN = os.path.join(HERE, "golden", "golden_seo.npz")


@pytest.fixture(scope="module")
def gs():
    z = np.load(GOLDEN)
    return {k: z[k] for k in z.files}


def _gp(gs, key):
    cfg = json.loads(bytes(gs[key + "_cfg"]).decode())
    gp = FFAG_GlobalParameters()
    gp.AddBMap(FFAG_Bfield_analytical(config=cfg, max_order=0, AddNumricalMap=False))
    return gp


def _golden_table(gs, key):
    lines = bytes(gs[key + "_ini"]).decode().splitlines()
    return lines, np.array([[float(v) for v in ln.split()] for ln in lines[1:]])


def _check(res, gs, key, r_tol):
    lines, ref = _golden_table(gs, key)
    t = res["table"].copy()
    t[:, 2:6] = np.round(t[:, 2:6], 3)
    t[:, 6:] = np.round(t[:, 6:], 8)
    # rounded like the file: equal, or one unit in the last kept decimal
    assert np.all(np.abs(t[:, 2:6] - ref[:, 2:6]) <= 1.0001e-3), (t[:, 2:6], ref[:, 2:6])
    assert np.all(np.abs(t[:, 6:] - ref[:, 6:]) <= 1.0001e-8 * np.maximum(1, np.abs(ref[:, 6:]))), \
        (t[:, 6:] - ref[:, 6:])
    assert np.array_equal(t[:, :2], ref[:, :2])
    gr, gpr = gs[key + "_r"], gs[key + "_pr"]
    np.testing.assert_allclose(res["fi"], gr[0, 1:], rtol=0, atol=1e-15)
    assert np.abs(res["r"] - gr[1:, 1:]).max() <= r_tol
    assert np.abs(res["pr"] - gpr[1:, 1:]).max() <= r_tol


@pytest.mark.parametrize("key", ["flat", "spiral"])
def test_search_with_oracle_tracker_matches_reference(gs, key):
    gp = _gp(gs, key)
    finder = S.FFAG_SearchSEO(gp, tracker=O.ThetaTracker(gp.Bmap, gp.q))
    res = finder.search(gs[key + "_Ek"])
    _check(res, gs, key, 1e-9)


def test_seo_ini_text_format(gs):
    lines, ref = _golden_table(gs, "flat")
    text = S.format_seo_ini(ref, "X", 0.001)
    assert text.splitlines()[1:] == lines
    assert text.splitlines()[0] == "Bmap foldname=X, step h = 0.001000 rad"


def test_load_seo_params_roundtrip(gs):
    d = tempfile.mkdtemp()
    fold = os.path.join(d, "seo")
    os.makedirs(fold)
    _, ref = _golden_table(gs, "flat")
    Ek = gs["flat_Ek"]
    S.write_seo_files(fold, d, 0.001, ref, gs["flat_r"][0, 1:], Ek, gs["flat_r"][1:, 1:], gs["flat_pr"][1:, 1:])
    inj, path, data = S.LoadSEOParams(os.path.join(fold, "SEO_ini.txt"), 315.0)
    assert path == d
    w = (315.0 - Ek[0]) / (Ek[1] - Ek[0])
    np.testing.assert_allclose(inj[1], ref[0, 6] + w * (ref[1, 6] - ref[0, 6]), rtol=1e-15)
    np.testing.assert_allclose(inj[3], 1 / ref[0, 4] + w * (1 / ref[1, 4] - 1 / ref[0, 4]), rtol=1e-15)
    r = np.loadtxt(os.path.join(fold, "SEO_r.txt"), skiprows=1)
    np.testing.assert_array_equal(r, gs["flat_r"])


def _check_twiss(gs, key, tracker_factory):
    gp = _gp(gs, key)
    d = tempfile.mkdtemp()
    fold = os.path.join(d, "seo")
    os.makedirs(fold)
    lines, ref = _golden_table(gs, key)
    Ek = gs[key + "_Ek"]
    S.write_seo_files(fold, d, 0.001, ref, gs[key + "_r"][0, 1:], Ek, gs[key + "_r"][1:, 1:],
                      gs[key + "_pr"][1:, 1:])
    S.CalcBetaFunc(fold, Ek, gp, tracker=tracker_factory(gp))
    for name, tol in (("BetaFuncR", 1e-6), ("BetaFuncZ", 1e-6), ("AlphaFuncR", 1e-6), ("AlphaFuncZ", 1e-6),
                      ("Bz", 1e-12), ("Br", 1e-12), ("Bf", 1e-12)):
        got = np.loadtxt(os.path.join(fold, name + ".txt"), skiprows=1)
        want = gs[f"{key}_{name}"]
        assert got.shape == want.shape, name
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[:, 0], want[:, 0])
        scale = np.abs(want[1:, 1:]).max()
        assert np.abs(got[1:, 1:] - want[1:, 1:]).max() <= tol * scale, (name, np.abs(got - want).max())


@pytest.mark.parametrize("key", ["flat", "spiral"])
def test_twiss_with_oracle_tracker_matches_reference(gs, key):
    _check_twiss(gs, key, lambda gp: O.ThetaTracker(gp.Bmap, gp.q))


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["flat", "spiral"])
def test_gpu_twiss_matches_reference(gs, key):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    _check_twiss(gs, key, lambda gp: S.ThetaTracker(gp.Bmap, gp.q))


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["flat", "spiral"])
def test_gpu_search_matches_reference(gs, key):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    res = S.FFAG_SearchSEO(_gp(gs, key)).search(gs[key + "_Ek"])
    _check(res, gs, key, 1e-9)


@pytest.mark.gpu
def test_gpu_theta_tracks_match_oracle(gs):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    gp = _gp(gs, "spiral")
    from pyffa_b200.constants import FFAG_ConversionTools
    rng = np.random.Generator(np.random.PCG64(5))
    m = 64
    P = FFAG_ConversionTools().Ek2P(300.0 + 20.0 * rng.random(m))
    x0 = np.stack([8.2 + 0.05 * rng.standard_normal(m), 0.1 + 0.01 * rng.standard_normal(m),
                   1e-3 * rng.standard_normal(m), 1e-3 * rng.standard_normal(m), P], axis=1)
    for mode in (0, 1):
        for cols in (2, 7):
            g1, gt, _ = S.ThetaTracker(gp.Bmap, gp.q).run(x0, np.pi / 6, 0.001, mode, True, cols)
            o1, ot, _ = O.ThetaTracker(gp.Bmap, gp.q).run(x0, np.pi / 6, 0.001, mode, True, cols)
            assert np.abs(g1 - o1).max() <= 1e-12 * np.abs(o1).max()
            for c in range(cols):
                assert np.abs(gt[..., c] - ot[..., c]).max() <= 1e-12 * np.abs(ot[..., c]).max(), (mode, c)
