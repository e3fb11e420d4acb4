"""Physical constants, the particle-matrix column map and the p/v-format
conversions of the tracking boundary.

Mirrors FFAG_GlobalParameters / FFAG_ConversionTools
(src/FFAG_ParasAndConversion.py:4-333) and FFAG_ManageBunchAttribute
(src/FFAG_Bunch.py:23-74).  The constants and conversion formulas have to be
the reference's own values and operation order: they define the on-disk
checkpoint format and the initial state both implementations start from.
"""
from __future__ import annotations

import numpy as np

# column map of the N x 16 particle matrix (src/FFAG_Bunch.py:23-74)
COLUMNS = {
    "r": 0, "vr": 1, "z": 2, "vz": 3, "fi": 4, "Ek": 5, "inj_t": 6, "Inj_flag": 7,
    "Survive": 8, "RF_phase": 9, "Esc_r": 10, "Esc_z": 11, "Esc_fi": 12,
    "Bunch_ID": 13, "Local_ID": 14, "Global_ID": 15,
}
NCOL = 16

Q = 1.60217662e-19          # C
C_LIGHT = 2.99792458e8      # m/s
E0_J = 938.2723e6 * Q       # proton rest energy, J
M0 = E0_J / C_LIGHT ** 2    # kg
E0_MEV = 938.2723


class FFAG_ManageBunchAttribute:
    """Column indices of the particle matrix (src/FFAG_Bunch.py:23-74)."""

    def __init__(self):
        self.Attribute = dict(COLUMNS)

    def get_num_attributes(self):
        return len(self.Attribute)

    def get_attribute_names(self):
        return list(self.Attribute.keys())


class FFAG_GlobalParameters:
    """Constants and the field / aperture registry passed to the pushers
    (src/FFAG_ParasAndConversion.py:4-81)."""

    def __init__(self):
        self.Bmap = None
        self.Emap = None
        self.Bunch = None
        self.SEOInfo = None
        self.q = Q
        self.c = C_LIGHT
        self.E0 = E0_J
        self.m0 = self.E0 / self.c ** 2
        self.ReverseTrack = False
        self.DumpInfo = None
        self.Aperture_m = None
        self.Aperture_enable = False
        self.BHarmonics = None

    def AddBMap(self, bmap):
        self.Bmap = bmap

    def AddEMap(self, emap):
        self.Emap = emap

    def AddBunch(self, bunch):
        self.Bunch = bunch

    def AddSEOInfo(self, seo):
        self.SEOInfo = seo

    def AddBHarmonics(self, harmonics):
        self.BHarmonics = harmonics

    def AddDumpInfo(self, dump):
        self.DumpInfo = dump

    def AddAperture(self, rmin, rmax, zmin, zmax):
        self.Aperture_m = np.array((rmin, rmax, zmin, zmax))
        self.Aperture_enable = True


class FFAG_ConversionTools:
    """p-format (r, pr=atan(vr/vf), z, pz, fi, Ek[MeV], ...) <-> v-format
    (src/FFAG_ParasAndConversion.py:84-333)."""

    q = Q
    c = C_LIGHT
    E0 = E0_J

    def Ek2v(self, Ek_value):
        Ek_J = Ek_value * 1e6 * self.q
        gamma = (Ek_J + self.E0) / self.E0
        beta = np.sqrt(1 - (1 / gamma) ** 2)
        return beta * self.c

    def Ek2P(self, Ek_value):
        Ek_J = Ek_value * 1e6 * self.q
        return 1 / self.c * np.sqrt((Ek_J + self.E0) ** 2 - self.E0 ** 2)

    def EkMeV2EtotJ(self, Ek_value):
        return Ek_value * 1e6 * self.q + self.E0

    def EtotJ2EkMeV(self, Etot_J):
        return (Etot_J - self.E0) / 1e6 / self.q

    def v2Ek(self, v):
        beta = v / self.c
        gamma = 1 / np.sqrt(1 - beta ** 2)
        return (gamma - 1) * self.E0 / 1e6 / self.q

    def _to_v(self, a, fifth):
        a = np.asarray(a, dtype=np.float64)
        v_c = self.Ek2v(a[:, 5])
        vr_rel = np.tan(a[:, 1]) * 1.0
        vz_rel = np.tan(a[:, 3]) * 1.0
        vtot = np.sqrt(vz_rel ** 2 + vr_rel ** 2 + 1.0 ** 2)
        vr = v_c * (vr_rel / vtot)
        vz = v_c * (vz_rel / vtot)
        vf = v_c * (1.0 / vtot)
        col5 = vf / a[:, 0] if fifth == "dfdt" else self.EkMeV2EtotJ(a[:, 5])
        return np.column_stack((a[:, 0], vr, a[:, 2], vz, a[:, 4], col5, a[:, 6], a[:, 7], a[:, 8], a[:, 9],
                                a[:, 10], a[:, 11], a[:, 12], a[:, 13], a[:, 14], a[:, 15]))

    def ConvertPrzek2Vrzek_boris(self, all_points):
        """p-format -> Boris v-format (col 5 = dfi/dt), src/FFAG_ParasAndConversion.py:202-234."""
        return self._to_v(all_points, "dfdt")

    def ConvertPrzek2Vrzek(self, all_points):
        """p-format -> RK4 v-format (col 5 = Etot [J]), src/FFAG_ParasAndConversion.py:237-269."""
        return self._to_v(all_points, "etot")

    def ConvertVrzek2Przek_boris(self, all_points):
        """Boris v-format -> p-format, src/FFAG_ParasAndConversion.py:272-301."""
        a = np.asarray(all_points, dtype=np.float64)
        vf = a[:, 5] * a[:, 0]
        v_c = np.sqrt(a[:, 1] ** 2 + a[:, 3] ** 2 + vf ** 2)
        ek = self.v2Ek(v_c)
        vr_d = a[:, 1] / v_c
        vz_d = a[:, 3] / v_c
        vf_d = np.sqrt(1 - vr_d ** 2 - vz_d ** 2)
        pr = np.arctan2(vr_d, vf_d)
        pz = np.arctan2(vz_d, vf_d)
        return np.column_stack((a[:, 0], pr, a[:, 2], pz, a[:, 4], ek, a[:, 6], a[:, 7], a[:, 8], a[:, 9],
                                a[:, 10], a[:, 11], a[:, 12], a[:, 13], a[:, 14], a[:, 15]))

    def ConvertVrzek2Przek(self, all_points):
        """RK4 v-format -> p-format, src/FFAG_ParasAndConversion.py:304-333."""
        a = np.asarray(all_points, dtype=np.float64)
        ek = self.EtotJ2EkMeV(a[:, 5])
        v_c = self.Ek2v(ek)
        vr_d = a[:, 1] / v_c
        vz_d = a[:, 3] / v_c
        vf_d = np.sqrt(1 - vr_d ** 2 - vz_d ** 2)
        pr = np.arctan2(vr_d, vf_d)
        pz = np.arctan2(vz_d, vf_d)
        return np.column_stack((a[:, 0], pr, a[:, 2], pz, a[:, 4], ek, a[:, 6], a[:, 7], a[:, 8], a[:, 9],
                                a[:, 10], a[:, 11], a[:, 12], a[:, 13], a[:, 14], a[:, 15]))
