"""The RF-bucket-matched longitudinal distribution (FFAG_bucket,
src/FFAG_bucket.py; the 'match' type of src/FFAG_Distribution.py:1270-1275)
against the reference's own bucket on the same closed-orbit table
(tests/golden/make_golden.py --bucket): starting points, stability flags
and box limits exactly; the trajectories' end points, the H grid, the
centre-line H-span relation and the thresholds to 1e-9 (the reference's
derivative is Numba-compiled, its sines may round differently from numpy's
over 18000 RK4 steps); the accepted sample in distribution (the reference
draws unseeded)."""
import os
import tempfile

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden_bucket.npz")


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def folder(gold):
    d = tempfile.mkdtemp()
    os.makedirs(os.path.join(d, "resultsSEO"))
    with open(os.path.join(d, "resultsSEO", "SEO_ini.txt"), "w") as f:
        f.write(bytes(gold["seo_ini_text"]).decode())
    return d


@pytest.mark.parametrize("k", [0, 1])
def test_bucket_matches_reference(gold, folder, k):
    from pyffa_b200.bucket import FFAG_bucket
    fi0, U0, Tc, w0, zd_u = gold[f"b{k}_params"]
    b = FFAG_bucket(folder, Ek0=300.0, fi0=fi0, U0=U0, step_t=20e-9, step_N=18000)
    assert (b.Tc, b.w0, b.zd_u) == (Tc, w0, zd_u)
    assert np.array_equal(b.X_in, gold[f"b{k}_X_in"])
    assert np.array_equal(np.stack([b.stable_fwd, b.stable_rev]), gold[f"b{k}_stable"])
    ends = np.stack([b.tr_fwd[-1], b.tr_rev[-1]])
    ref_ends = gold[f"b{k}_tr_end"]
    scale = np.abs(ref_ends).max(axis=(0, 1), keepdims=True)
    assert np.all(np.abs(ends - ref_ends) <= 1e-9 * scale)
    lim = np.array([b.x_min_plot, b.x_max_plot, b.y_min_plot, b.y_max_plot,
                    b.x_min_sample, b.x_max_sample, b.y_min_sample, b.y_max_sample])
    np.testing.assert_allclose(lim, gold[f"b{k}_limits"], rtol=1e-9, atol=1e-9)
    b.build_H()
    for got, ref in zip((b.q_grid, b.p_grid, b.Hq_rel, b.Hp_rel), gold[f"b{k}_H"]):
        np.testing.assert_allclose(got, ref, rtol=1e-8, atol=1e-9 * np.abs(ref).max())
    H, L = b.compute_center_H_vs_span()
    np.testing.assert_allclose(np.stack([H, L]), gold[f"b{k}_HL"], rtol=1e-8, atol=1e-12)
    thr = [b.threshold(Lt) for Lt in (30.0, 80.0, 1e4)]
    np.testing.assert_allclose(thr, gold[f"b{k}_thr"], rtol=1e-8, atol=1e-12)
    # the accepted draw: same region, same moments within sampling error
    t, E, H_thr = b.scatter_filter_by_span(20000, 80.0, rng=np.random.default_rng(3))
    ref = gold[f"b{k}_sample"]
    assert len(t) == 20000 and np.all(b.H_at(t * 1e-9, E - b.E0) >= H_thr)
    for a, r in ((t, ref[:, 0]), (E, ref[:, 1])):
        sd = r.std()
        assert abs(a.mean() - r.mean()) <= 6 * sd / np.sqrt(len(r))
        assert abs(a.std() / sd - 1) <= 0.05
