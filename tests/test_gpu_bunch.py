"""The GPU bunch generator (ffa_bunch_sample, the device path of
GenerateBunches; src/FFAG_Distribution.py:1152-1741).

Against the oracle's numpy restatement (oracle/bunch.py): every row equal to
rounding (the Philox integers are exact; sin / cos / log / sqrt of the two
sides differ by an ulp or so), identifiers exact.  The draw depends only on
(seed, sub-bunch, particle id, draw group): two calls give the same rows,
and a bunch drawn in two calls equals the one drawn in one.  The whole
painted bunch on the device against the bunches the reference generated
(tests/golden/golden_bunch.npz): the same agreement in distribution as the
host generator's."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TW = ((-0.8, 2.5, 1.2e-6), (0.4, 5.0, 0.7e-6), (0.1, 40.0, 3e-3))
CENTRE = (8.5, 0.01, 1e-4, -2e-4, 300.0, 5.0)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _gpu(n, seed, sub, tt, lt, id0=0, out=None):
    from pyffa_b200 import distribution as D
    out = torch.empty((n, 16), dtype=torch.float64, device="cuda") if out is None else out
    D._sample_on_device(out, n, tt, lt, TW, 100.0, 0.05, CENTRE, 0.2, sub, seed, id0=id0)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("tt,lt", [("gauss", "gauss"), ("kv", "kv"), ("waterbag", "waterbag"),
                                   ("hollow_waterbag", "hollow_waterbag"), ("kv", "UniformGauss")])
def test_rows_match_oracle(tt, lt):
    from oracle import bunch as OB
    from pyffa_b200 import _lib
    n = 100_000
    got = _gpu(n, 1234567, 5, tt, lt).cpu().numpy()
    ref = OB.sample(n, 1234567, 5, _lib.DIST_TYPES[tt], _lib.DIST_TYPES[lt], TW, CENTRE, 0.2, 5.0,
                    uniform_length=100.0, uniform_sigma=0.05)
    for c in (4, 7, 8, 9, 10, 11, 12, 13, 14, 15):
        assert np.array_equal(got[:, c], ref[:, c]), c
    for c in (0, 1, 2, 3, 5, 6):
        dev = ref[:, c] - CENTRE[c if c < 4 else (4 if c == 5 else 5)]
        scale = np.abs(dev).max()
        assert np.abs(got[:, c] - ref[:, c]).max() <= 1e-12 * scale + 1e-15 * np.abs(ref[:, c]).max(), c


def test_reproducible_and_split_invariant():
    n = 65_537
    a = _gpu(n, 99, 0, "waterbag", "gauss").cpu().numpy()
    b = _gpu(n, 99, 0, "waterbag", "gauss").cpu().numpy()
    assert np.array_equal(a, b)
    whole = torch.empty((n, 16), dtype=torch.float64, device="cuda")
    h = 30_001
    _gpu(h, 99, 0, "waterbag", "gauss", id0=0, out=whole[:h])
    _gpu(n - h, 99, 0, "waterbag", "gauss", id0=h, out=whole[h:])
    assert np.array_equal(whole.cpu().numpy(), a)
    c = _gpu(n, 99, 1, "waterbag", "gauss").cpu().numpy()
    assert not np.array_equal(a[:, 0], c[:, 0])


@pytest.mark.parametrize("key", ["paint", "kv"])
def test_painted_bunch_on_device_matches_reference_in_distribution(key):
    import os
    from pyffa_b200 import distribution as D
    from tests.test_distribution import GOLDEN
    z = np.load(GOLDEN)
    g = {k: z[k] for k in z.files}
    import tempfile
    d = tempfile.mkdtemp()
    fold = os.path.join(d, "seo")
    os.makedirs(fold)
    for name in ("SEO_ini", "SEO_r", "SEO_pr", "BetaFuncR", "BetaFuncZ", "AlphaFuncR", "AlphaFuncZ"):
        with open(os.path.join(fold, name + ".txt"), "w") as f:
            f.write(bytes(g["file_" + name]).decode())
    for name, fn in (("emap", "emap.txt"), ("paint", "paint.txt")):
        with open(os.path.join(d, fn), "w") as f:
            f.write(bytes(g["file_" + name]).decode())
    para = json.loads(bytes(g[key + "_para"]).decode())
    para.update(SEO=fold, BmapPATHName=d, PaintCurve=os.path.join(d, "paint.txt"),
                EmapPATHName=os.path.join(d, "emap.txt"), Seed=11)
    mine = D.GenerateBunches(para, device="cuda").cpu().numpy()
    ref = g[key + "_bunch"]
    assert mine.shape == ref.shape
    np.testing.assert_array_equal(mine[:, 13], ref[:, 13])
    np.testing.assert_array_equal(mine[:, 14], ref[:, 14])
    np.testing.assert_array_equal(mine[:, 4], ref[:, 4])
    assert not mine[:, 7:13].any()
    for b in np.unique(ref[:, 13]):
        m, r = mine[mine[:, 13] == b], ref[ref[:, 13] == b]
        n = len(r)
        for c in (0, 1, 2, 3, 5, 6):
            sd = r[:, c].std()
            assert abs(m[:, c].mean() - r[:, c].mean()) <= 6 * sd / np.sqrt(n) + 1e-15, (b, c)
            assert abs(m[:, c].std() / sd - 1) <= 0.06, (b, c)
