"""Loads tests/golden/golden_tracking.npz into the product's host objects.

The fixture holds every input the reference was run on (lattice JSON,
z-Taylor stacks, RF file text, closed-orbit tables, particle matrices) and
the reference's outputs; see tests/golden/make_golden.py."""
from __future__ import annotations

import io
import json
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "golden_tracking.npz")
GOLDEN_HARMONICS = os.path.join(HERE, "golden", "golden_harmonics.npz")
GOLDEN_SPIRAL = os.path.join(HERE, "golden", "golden_spiral.npz")


class Golden:
    def __init__(self, path=GOLDEN):
        z = np.load(path)
        self.z = {k: z[k] for k in z.files}
        self.cfg = json.loads(bytes(self.z["cfg_json"]).decode())
        self.emap_text = bytes(self.z["emap_text"]).decode()
        self.aperture = tuple(self.z["aperture"].tolist())
        self.seo = {k: self.z["seo_" + k] for k in ("Ek_axis", "fi_axis", "r", "pr", "perimeter")}

    def __getitem__(self, k):
        return self.z[k]

    def bmap(self, max_order=2):
        from pyffa_b200.fields import FFAG_Bfield_analytical
        st = tuple(np.concatenate([np.zeros_like(self.z[k][:1]), self.z[k]])
                   for k in ("stack_Bz", "stack_Bfi", "stack_Br"))
        return FFAG_Bfield_analytical(config=self.cfg, max_order=max_order, stacks=st)

    def emap(self, enable=True):
        from pyffa_b200.fields import FFAG_EField_new, parse_emap_file
        with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
            f.write(self.emap_text)
            p = f.name
        try:
            h, d = parse_emap_file(p)
        finally:
            os.unlink(p)
        return FFAG_EField_new(header=h, data=d, EnableFlag=enable)

    def gp(self, aperture=True):
        from pyffa_b200.constants import FFAG_GlobalParameters
        from pyffa_b200.fields import FFAG_BField_Error
        g = FFAG_GlobalParameters()
        g.AddBMap(self.bmap())
        g.AddEMap(self.emap())
        if aperture:
            g.AddAperture(*self.aperture)
        if "harmonics_json" in self.z:
            g.AddBHarmonics(FFAG_BField_Error(json.loads(bytes(self.z["harmonics_json"]).decode()), True))
        return g


class SpiralGolden(Golden):
    """The spiral-gap fixture (tests/golden/make_golden.py --spiral): the
    tracking fixture's lattice with the spiral RF gap files it stores."""

    def __init__(self, path=None):
        z = np.load(path or GOLDEN_SPIRAL)
        self.z = {k: z[k] for k in z.files}
        self.cfg = json.loads(bytes(self.z["cfg_json"]).decode())
        self.aperture = tuple(self.z["aperture"].tolist())
        self.folder = tempfile.mkdtemp()
        for name in ("emap", "Er_coef", "Ez_coef", "Ephi_coef"):
            with open(os.path.join(self.folder, name + ".txt"), "w") as f:
                f.write(bytes(self.z["file_" + name]).decode())

    def emap(self, enable=True):
        from pyffa_b200.fields import FFAG_EField_spiral
        return FFAG_EField_spiral(os.path.join(self.folder, "emap.txt"), enable)


_cache = {}


def load_golden():
    if "g" not in _cache:
        _cache["g"] = Golden()
    return _cache["g"]


def load_golden_harmonics():
    """The harmonics fixture: the tracking fixture's lattice with field-error
    harmonics enabled (FFAG_BField_Error), single steps and loops."""
    if "h" not in _cache:
        _cache["h"] = Golden(GOLDEN_HARMONICS)
    return _cache["h"]


def load_golden_spiral():
    """The spiral RF gap fixture: field lookups, single steps and loops."""
    if "s" not in _cache:
        _cache["s"] = SpiralGolden()
    return _cache["s"]


def rel_err(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if scale is None:
        scale = np.maximum(np.abs(b), 1e-300)
    return np.max(np.abs(a - b) / scale) if a.size else 0.0
