"""Injected-bunch generation (GenerateBunches, src/FFAG_Distribution.py:1542-1741).

tests/golden/golden_bunch.npz holds the reference's SEO and Twiss tables for
the synthetic lattice (290-320 MeV), its injection point and Twiss at
injection, and two bunches it generated with seeded global random streams
(tests/golden/make_golden.py --bunch).  The deterministic helpers must agree
to rounding; the bunches, drawn from a different random stream, must agree
in distribution."""
import json
import os
import tempfile

import numpy as np
import pytest

from pyffa_b200 import distribution as D

from .fixtures import HERE

GOLDEN = os.path.join(HERE, "golden", "golden_bunch.npz")


@pytest.fixture(scope="module")
def gb():
    z = np.load(GOLDEN)
    g = {k: z[k] for k in z.files}
    d = tempfile.mkdtemp()
    fold = os.path.join(d, "seo")
    os.makedirs(fold)
    for name in ("SEO_ini", "SEO_r", "SEO_pr", "BetaFuncR", "BetaFuncZ", "AlphaFuncR", "AlphaFuncZ"):
        with open(os.path.join(fold, name + ".txt"), "w") as f:
            f.write(bytes(g["file_" + name]).decode())
    for name, fn in (("emap", "emap.txt"), ("paint", "paint.txt")):
        with open(os.path.join(d, fn), "w") as f:
            f.write(bytes(g["file_" + name]).decode())
    g["_fold"], g["_dir"] = fold, d
    return g


def test_injection_point_and_twiss(gb):
    SEO_R = np.loadtxt(os.path.join(gb["_fold"], "SEO_r.txt"), skiprows=1)
    SEO_Pr = np.loadtxt(os.path.join(gb["_fold"], "SEO_pr.txt"), skiprows=1)
    got = np.array(D.GetInitRAndFiForInjection(SEO_R, SEO_Pr, 7.5, 305.0))
    np.testing.assert_allclose(got, gb["inj_point"], rtol=1e-14)
    tw = np.array(D.LoadSEOBetaFunc(gb["_fold"], 305.0, float(got[0])))
    np.testing.assert_allclose(tw, gb["inj_twiss"], rtol=1e-13)


@pytest.mark.parametrize("kind", ["gauss", "kv", "waterbag"])
def test_transverse_rms_emittance_and_twiss(kind):
    rng = np.random.default_rng(3)
    tx, ty = D.TwissContainer(-0.8, 2.5, 1.2e-6), D.TwissContainer(0.4, 5.0, 0.7e-6)
    x, xp, y, yp = D.create_distribution(kind, twiss_transverse=(tx, ty)).sample(400_000, rng)
    for u, up, tw in ((x, xp, tx), (y, yp, ty)):
        u, up = u - u.mean(), up - up.mean()
        e = np.sqrt(np.mean(u * u) * np.mean(up * up) - np.mean(u * up) ** 2)
        assert abs(e / tw.emittance - 1) < 0.01
        assert abs(np.mean(u * u) / e / tw.beta - 1) < 0.01
        assert abs(-np.mean(u * up) / e - tw.alpha) < 0.02


@pytest.mark.parametrize("key", ["paint", "kv"])
def test_bunch_matches_reference_in_distribution(gb, key):
    para = json.loads(bytes(gb[key + "_para"]).decode())
    para.update(SEO=gb["_fold"], BmapPATHName=gb["_dir"], PaintCurve=os.path.join(gb["_dir"], "paint.txt"),
                EmapPATHName=os.path.join(gb["_dir"], "emap.txt"), Seed=11)
    mine = D.GenerateBunches(para)
    ref = gb[key + "_bunch"]
    assert mine.shape == ref.shape
    np.testing.assert_array_equal(mine[:, 13], ref[:, 13])       # Bunch_ID
    np.testing.assert_array_equal(mine[:, 14], ref[:, 14])       # Local_ID
    np.testing.assert_array_equal(mine[:, 4], ref[:, 4])         # injection azimuth
    assert not mine[:, 7:13].any() and not ref[:, 7:13].any()
    for b in np.unique(ref[:, 13]):
        m, r = mine[mine[:, 13] == b], ref[ref[:, 13] == b]
        n = len(r)
        for c in (0, 1, 2, 3, 5, 6):
            sd = r[:, c].std()
            assert abs(m[:, c].mean() - r[:, c].mean()) <= 6 * sd / np.sqrt(n) + 1e-15, (b, c)
            assert abs(m[:, c].std() / sd - 1) <= 0.06, (b, c)
