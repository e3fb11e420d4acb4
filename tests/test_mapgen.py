"""z-Taylor map generation (Generate_Bmaps, src/FFAG_HighOrder.py:828-998).

tests/golden/golden_mapgen.npz holds the reference's own tables for the
synthetic lattice and for the same lattice with a 35-degree spiral
(tests/golden/make_golden.py --mapgen).  The oracle restates the reference
term by term; the product factors every entry into r-only weights times
flutter derivatives and evaluates it on the GPU."""
import json
import os
import tempfile

import numpy as np
import pytest
from numpy.polynomial import Polynomial

from oracle import mapgen as M
from pyffa_b200 import mapgen as G

from .fixtures import HERE

GOLDEN = os.path.join(HERE, "golden", "golden_mapgen.npz")
NAMES = ("Bz", "Br", "Bfi")


@pytest.fixture(scope="module")
def gm():
    z = np.load(GOLDEN)
    return {k: z[k] for k in z.files}


def _setup(gm, key):
    B = json.loads(bytes(gm[key + "_cfg"]).decode())["Bmap"]
    r, fi = G.map_axes(B)
    sfit = Polynomial.fit(r, G.calculate_s(r, 0.0, B["SpiralAngle_deg"]), 5)
    return B, r, fi, sfit


def _rel(a, ref):
    return float(np.abs(a - ref).max() / np.abs(ref).max())


@pytest.mark.parametrize("key", ["flat", "spiral"])
def test_oracle_matches_reference_tables(gm, key):
    B, r, fi, sfit = _setup(gm, key)
    Br, Bz, Bfi = M.generate_bmaps(2, r, fi, M.convex_params(B), sfit, B["coefficients_tupel"])
    for name, mine in zip(("Br", "Bz", "Bfi"), (Br, Bz, Bfi)):
        for n in range(3):
            assert _rel(mine[n], gm[f"{key}_{name}"][n]) <= 1e-15, (name, n)


@pytest.mark.parametrize("key", ["flat", "spiral"])
def test_weight_factorisation_matches_reference(gm, key):
    """The product's host weights, combined with the oracle's flutter
    derivatives the way the kernel combines them, give the reference's
    tables (no GPU)."""
    B, r, fi, sfit = _setup(gm, key)
    conv = G.BmapParams_to_ConvexParams(B)
    W = G.weights(2, r, B["coefficients_tupel"], sfit)
    Gp = np.stack([M.flutter(fi, conv, p)[1] for p in range(W.shape[-1])])
    dth = fi[1] - fi[0]
    out = np.zeros((3, 3, len(r), len(fi)))
    for i, x in enumerate(r):
        out[:, :, i, :] = np.einsum("cnp,pj->cnj", W[:, :, i, :], np.roll(Gp, int(sfit(x) / dth), axis=1))
    out /= Gp[0].mean()
    for c, name in enumerate(NAMES):
        for n in range(3):
            assert _rel(out[c, n], gm[f"{key}_{name}"][n]) <= 4e-15, (name, n)


def test_chain_rule_terms():
    # d2/dr2 G(th - s(r)) = G'' s'^2 - G' s''
    assert G._chain(2) == {(2, (0, 2)): 1, (1, (0, 0, 1)): -1}
    # d3: -G''' s'^3 + 3 G'' s' s'' - G' s'''
    assert G._chain(3) == {(3, (0, 3)): -1, (2, (0, 1, 1)): 3, (1, (0, 0, 0, 1)): -1}


def test_sigmoid_polynomials():
    k = 3.7
    x = np.linspace(-2, 2, 41)
    s = 1 / (1 + np.exp(-k * x))
    P = G.sigmoid_polys(k, 4)
    ev = lambda row, n: np.polyval(row[:n], s)
    assert np.allclose(ev(P[0], 2), s)
    assert np.allclose(ev(P[1], 3), k * s * (1 - s))
    assert np.allclose(ev(P[2], 4), k * k * s * (1 - s) * (1 - 2 * s))


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["flat", "spiral"])
def test_gpu_tables_match_reference(gm, key):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    B, r, fi, sfit = _setup(gm, key)
    Br, Bz, Bfi = G.Generate_Bmaps(2, r, fi, G.BmapParams_to_ConvexParams(B), sfit, B["coefficients_tupel"])
    for name, mine in zip(("Br", "Bz", "Bfi"), (Br, Bz, Bfi)):
        for n in range(3):
            assert mine[n].shape == gm[f"{key}_{name}"][n].shape
            assert _rel(mine[n], gm[f"{key}_{name}"][n]) <= 1e-13, (name, n)


@pytest.mark.gpu
def test_gpu_full_grid_rows_match_oracle():
    """The workloads' 1301 x 6000 order-2 map: three rows of every table
    against the oracle (which evaluates rows independently)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from pyffa_b200 import synthetic
    cfg = synthetic.lattice_bmap()
    B = cfg["Bmap"]
    B["SpiralAngle_deg"] = 20.0
    r, fi = G.map_axes(B)
    assert (len(r), len(fi)) == (1301, 6000)
    sfit = Polynomial.fit(r, G.calculate_s(r, 0.0, 20.0), 5)
    conv = G.BmapParams_to_ConvexParams(B)
    t = G.generate_device(2, r, fi, conv, sfit, B["coefficients_tupel"]).cpu().numpy()
    rows = [0, 650, 1300]
    Br, Bz, Bfi = M.generate_bmaps(2, r[rows], fi, M.convex_params(B), sfit, B["coefficients_tupel"])
    for c, ref in enumerate((Bz, Br, Bfi)):
        for n in range(3):
            assert _rel(t[c, n, rows], ref[n]) <= 1e-13, (NAMES[c], n)


@pytest.mark.gpu
def test_gpu_main_bmap_writes_reference_files():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from pyffa_b200 import synthetic
    cfg = synthetic.lattice_bmap(r_range=(8.0, 8.2, 0.05), theta_step_deg=0.25)
    cfg["config"] = {"folder": "maps", "expand_order": 1}
    d = tempfile.mkdtemp()
    path = os.path.join(d, "config_Bmap.json")
    with open(path, "w") as f:
        json.dump(cfg, f)
    out = G.main_Bmap(path)
    assert out == os.path.join(d, "maps")
    r, fi = G.map_axes(cfg["Bmap"])
    for comp in ("Br", "Bz", "Bfi"):
        for n in range(2):
            a = np.load(os.path.join(out, f"{comp}_order_{n}.npz"))[f"{comp}_Taylor_coeff"]
            assert a.shape == (len(r), len(fi)) and np.isfinite(a).all()
