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


# ------------------------------------------------ the GPU generator's oracle

def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors (counter, key -> output) of its
    published description, through the oracle's restatement."""
    from oracle import bunch as OB
    M = 0xFFFFFFFF
    for ctr, key, want in (((0, 0, 0, 0), 0, (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
                           ((M, M, M, M), (M << 32) | M, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
                           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0x299f31d0 << 32) | 0xa4093822,
                            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))):
        got = [int(x) for x in OB.philox4x32_10(*ctr, key)]
        assert got == list(want)


@pytest.mark.parametrize("kind,ltype", [("gauss", "gauss"), ("kv", "kv"), ("waterbag", "waterbag"),
                                        ("hollow_waterbag", "hollow_waterbag"), ("gauss", "UniformGauss")])
def test_device_sampler_oracle_matches_host_generator_in_distribution(kind, ltype):
    """The restated device sampler (Philox draws) against the host numpy
    generator of the same shapes: means, rms sizes and rms emittances of
    every plane agree within sampling error."""
    from oracle import bunch as OB
    from pyffa_b200 import _lib
    tw = ((-0.8, 2.5, 1.2e-6), (0.4, 5.0, 0.7e-6), (0.1, 40.0, 3e-3))
    n = 200_000
    # the longitudinal emittance as GenerateInitDistributionDtInjNew hands it
    # to the shapes (doubled for KV)
    lt = tw[2][2] * (2 if ltype == "kv" else 1)
    got = OB.sample(n, 77, 3, _lib.DIST_TYPES[kind], _lib.DIST_TYPES[ltype], (tw[0], tw[1], (tw[2][0], tw[2][1], lt)),
                    (8.5, 0.01, 0.0, 0.0, 300.0, 5.0), 0.2, 3.0, uniform_length=100.0, uniform_sigma=0.05)
    dist = D.CustomDist3D(D.create_distribution(kind, twiss_transverse=(D.TwissContainer(*tw[0]),
                                                                        D.TwissContainer(*tw[1]))),
                          D.create_distribution(ltype, twiss_longitudinal=D.TwissContainer(tw[2][0], tw[2][1], lt)))
    r, pr, z, pz, t, E = dist.sample(n, np.random.default_rng(5))
    if ltype == "UniformGauss":
        t, E = np.random.default_rng(6).uniform(-50.0, 50.0, n), np.random.default_rng(7).normal(0.0, 0.05, n)
    ref = np.stack([r + 8.5, pr + 0.01, z, pz, E + 300.0, t + 5.0], 1)
    mine = got[:, [0, 1, 2, 3, 5, 6]]
    assert np.all(got[:, 4] == 0.2) and np.all(got[:, 13] == 3.0) and np.array_equal(got[:, 14], np.arange(n))
    for c in range(6):
        sd = ref[:, c].std()
        assert abs(mine[:, c].mean() - ref[:, c].mean()) <= 6 * sd / np.sqrt(n), c
        assert abs(mine[:, c].std() / sd - 1) <= 0.02, c
    for a, b in ((0, 1), (2, 3)):
        e = lambda m: np.sqrt(np.cov(m[:, a], m[:, b]).diagonal().prod() - np.cov(m[:, a], m[:, b])[0, 1] ** 2)
        assert abs(e(mine) / e(ref) - 1) <= 0.02


def test_central_line_injection_point_matches_reference_steps():
    """Injection along a central line (GetInitRAndFiForInjection, central-line
    branch, src/FFAG_Distribution.py:1361-1406) against the values the
    reference's own helpers give for 8 lines and energies
    (tests/golden/golden_injection.npz; the reference function itself raises
    at its last line, which the fixture records)."""
    import os
    from pyffa_b200.distribution import GetInitRAndFiForInjection
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_injection.npz"))
    assert int(z["reference_raised"][0]) == 8
    for k, (Ek, th, r, pr, i, j) in enumerate(z["cases"]):
        got = GetInitRAndFiForInjection(z["seo_r"], z["seo_pr"], z[f"line_{k}"], Ek)
        assert got == (th, r, pr), (k, got, (th, r, pr))


def test_central_line_file_in_the_generator(tmp_path):
    """A str InjectionPosition is read as a central-line file (x, y after one
    header line), as the reference's generator does."""
    import os
    from pyffa_b200.distribution import GetInitRAndFiForInjection
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_injection.npz"))
    p = tmp_path / "cl.txt"
    np.savetxt(p, z["line_0"], header="x y", comments="")
    line = np.loadtxt(str(p), skiprows=1)
    assert np.array_equal(line, z["line_0"])
    Ek = z["cases"][0, 0]
    assert GetInitRAndFiForInjection(z["seo_r"], z["seo_pr"], line, Ek) == tuple(z["cases"][0, 1:4])


def test_match_longitudinal_draws_inside_the_bucket(gb):
    """The 'match' longitudinal type (src/FFAG_Distribution.py:1270-1275):
    energies and times from the RF bucket's rejection draw for the target
    bunch length (FFAG_bucket, built from the closed-orbit table of the map
    folder's resultsSEO), transverse rows as for the other types."""
    import shutil
    from pyffa_b200.bucket import FFAG_bucket
    os.makedirs(os.path.join(gb["_dir"], "resultsSEO"), exist_ok=True)
    shutil.copy(os.path.join(gb["_fold"], "SEO_ini.txt"), os.path.join(gb["_dir"], "resultsSEO", "SEO_ini.txt"))
    rng = np.random.default_rng(7)
    a, _, centre, bucket = D.GenerateInitDistributionDtInjNew(
        gb["_fold"], 0.0, 300.0, (1.0, 1.0, 1e-3), 4000, 5.0, 0.0, 40.0, 60.0, acc_U0=100e3, acc_phi0=30.0,
        dist_types=("gauss", "match"), rng=rng)
    assert isinstance(bucket, FFAG_bucket)
    Ek_c = centre[4]
    t, E = a[:, 6] - 5.0, a[:, 5]
    thr = bucket.threshold(60.0)
    assert np.all(bucket.H_at(t * 1e-9, E - Ek_c) >= thr - 1e-12 * abs(thr))
    assert bucket.x_min_sample <= t.min() and t.max() <= bucket.x_max_sample
    assert bucket.y_min_sample <= E.min() and E.max() <= bucket.y_max_sample
    assert a[:, 0].std() > 0 and np.all(a[:, 13] == 0)
