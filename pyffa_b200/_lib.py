"""ctypes binding of libffa_cuda.so (include/ffa_cuda.h).

The library is loaded from the package directory.  There is no fallback: if
the shared object is missing or fails to load, every GPU entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB_PATH

MAX_POLY = 16
MAX_SEG = 16
MAX_GAPS = 8
MAX_ORDER = 4

FFA_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA runtime error", 3: "out of device memory", 4: "unsupported"}

FFA_BORIS = 0
FFA_RK4 = 1
FFA_FP64 = 0
FFA_FP32C = 2
FFA_FP32 = 8
FFA_RF_PHYSICAL_SUM = 4
FFA_SHAPE_TB_SHIFT = 8
FFA_SHAPE_NREG_SHIFT = 10
FFA_SHAPE_MASK = 0xF00
SHAPE_THREADS = (32, 64, 128, 256)   # threads per block, bits 8-9
SHAPE_NREGS = (80, 72, 64, 56)       # register cap per thread, bits 10-11


def shape_flags(tb_sel: int, nreg_sel: int) -> int:
    """ffa_push flag bits of a Boris launch shape (0, 0: the default)."""
    if not (0 <= tb_sel < 4 and 0 <= nreg_sel < 4):
        raise ValueError(f"launch shape ({tb_sel}, {nreg_sel}) out of range")
    return (tb_sel << FFA_SHAPE_TB_SHIFT) | (nreg_sel << FFA_SHAPE_NREG_SHIFT)

STATUS_LOST = 0
STATUS_NAN = 1
STATUS_OUT_OF_MAP = 2
STATUS_SC_DEGENERATE = 3
STATUS_WORDS = 8

d_p = C.c_void_p  # device pointers travel as integers


class FieldDesc(C.Structure):
    _fields_ = [
        ("nsectors", C.c_int32), ("n_spoly", C.c_int32), ("n_spolyp", C.c_int32),
        ("n_convex", C.c_int32), ("max_order", C.c_int32), ("pad0", C.c_int32),
        ("B0", C.c_double), ("k", C.c_double),
        ("spoly", C.c_double * MAX_POLY), ("spolyp", C.c_double * MAX_POLY),
        ("convex", C.c_double * (MAX_SEG * 5)),
        ("r_min", C.c_double), ("r_step", C.c_double), ("r_size", C.c_int64),
        ("fi_min", C.c_double), ("fi_step", C.c_double), ("fi_size", C.c_int64),
        ("bz_stack", d_p), ("bfi_stack", d_p), ("br_stack", d_p),
    ]


class RFDesc(C.Structure):
    _fields_ = [
        ("enable", C.c_int32), ("ngaps", C.c_int32), ("pad0", C.c_int32), ("pad1", C.c_int32),
        ("poly_x", (C.c_double * 4) * MAX_GAPS), ("poly_y", (C.c_double * 4) * MAX_GAPS),
        ("box", (C.c_double * 4) * MAX_GAPS),
        ("theta_n", C.c_double * MAX_GAPS), ("rf_shift", C.c_double * MAX_GAPS),
        ("spiral_nodes", d_p), ("spiral_nr", C.c_int32), ("spiral_nphi", C.c_int32),
        ("spiral_r0", C.c_double), ("spiral_dr", C.c_double), ("spiral_phi0", C.c_double),
        ("spiral_dphi", C.c_double), ("gap_azimuth", C.c_double * MAX_GAPS),
    ]


class Aperture(C.Structure):
    _fields_ = [("enable", C.c_int32), ("pad0", C.c_int32),
                ("rmin", C.c_double), ("rmax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double)]


class Consts(C.Structure):
    _fields_ = [("q", C.c_double), ("c", C.c_double), ("m0", C.c_double), ("E0", C.c_double)]


class StateSoA(C.Structure):
    _fields_ = [
        ("r", d_p), ("vr", d_p), ("z", d_p), ("vz", d_p), ("fi", d_p), ("f5", d_p), ("rf", d_p),
        ("esc_r", d_p), ("esc_z", d_p), ("esc_fi", d_p),
        ("inj", d_p), ("surv", d_p), ("inj_step", d_p),
        ("e_pre_r", d_p), ("e_pre_z", d_p), ("e_pre_fi", d_p),
        ("e_pp_r", d_p), ("e_pp_z", d_p), ("e_pp_fi", d_p),
        ("sc_pre", d_p), ("sc_pp", d_p), ("order", d_p),
    ]


_SOA_ELEM = {"inj": 1, "surv": 1, "sc_pre": 1, "sc_pp": 1, "inj_step": 4}   # bytes; the rest float64


def soa_offset(st: "StateSoA", start: int) -> "StateSoA":
    """The SoA view of particles start.. of `st` (every non-null column
    pointer advanced by start elements)."""
    out = StateSoA()
    for name, _ in StateSoA._fields_:
        if name == "order":         # a permutation of the whole range: not carried over
            continue
        p = getattr(st, name)
        setattr(out, name, None if not p else p + start * _SOA_ELEM.get(name, 8))
    return out


class StepTable(C.Structure):
    _fields_ = [("drf", d_p), ("acc", d_p), ("nsteps", C.c_int64)]


CROSSING_RECORD = 23
MAX_CROSSING_TARGETS = 8


FIT_SUMS = 25


class Crossing(C.Structure):
    _fields_ = [("ntargets", C.c_int32), ("pad", C.c_int32), ("target", C.c_double * MAX_CROSSING_TARGETS),
                ("buf", d_p), ("capacity", C.c_int64), ("count", d_p),
                ("fit_instance", d_p), ("fit_centre", d_p), ("fit_scale", d_p), ("fit_last", d_p),
                ("fit_has", d_p), ("fit_sums", d_p)]


class ThetaTrackDesc(C.Structure):
    _fields_ = [("m", C.c_int64), ("n_points", C.c_int32), ("time_mode", C.c_int32), ("traj_cols", C.c_int32),
                ("pad", C.c_int32), ("t_end", C.c_double),
                ("q", C.c_double), ("x0", d_p), ("x1", d_p), ("traj", d_p)]


MAPGEN_MAX_DERIV = 16


class MapgenDesc(C.Structure):
    _fields_ = [("n_seg", C.c_int32), ("n_deriv", C.c_int32), ("n_orders", C.c_int32), ("pad", C.c_int32),
                ("n_r", C.c_int64), ("n_theta", C.c_int64),
                ("seg_x0", C.c_double * MAX_SEG), ("seg_x1", C.c_double * MAX_SEG),
                ("seg_k", C.c_double * MAX_SEG), ("seg_y", C.c_double * MAX_SEG),
                ("sig_poly", d_p), ("theta", d_p), ("weights", d_p), ("shift", d_p),
                ("gder", d_p), ("gmean", d_p), ("bz", d_p), ("br", d_p), ("bfi", d_p)]


MLP_HIDDEN = 256
MLP_PARAMS = 138192
MLP_WPACK_BYTES = 278528
MLP_SPLIT_WORK = 1048576


class MlpTrainDesc(C.Structure):
    _fields_ = [("batch", C.c_int64), ("n_fit", C.c_int32), ("step", C.c_int32),
                ("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("params", d_p), ("grads", d_p), ("adam_m", d_p), ("adam_v", d_p), ("mask", d_p),
                ("x", d_p), ("target", d_p), ("work", d_p), ("loss_part", d_p),
                ("lr_table", d_p), ("counter", d_p)]


class MlpInferDesc(C.Structure):
    _fields_ = [("n", C.c_int64), ("n_apply", C.c_int32), ("radius2", C.c_float),
                ("params", d_p), ("wpack", d_p), ("state", d_p), ("applied", d_p), ("error", d_p)]


class SCDesc(C.Structure):
    _fields_ = [
        ("ns", C.c_int32), ("nx", C.c_int32), ("nz", C.c_int32), ("hockney", C.c_int32),
        ("boris", C.c_int32), ("pad0", C.c_int32), ("n_max", C.c_int64),
        ("sigma_ratio", C.c_double), ("q_macro", C.c_double),
        ("speed_c", C.c_double), ("E0_rest_MeV", C.c_double), ("E0_J", C.c_double),
        ("nE", C.c_int64), ("nfi", C.c_int64),
        ("Ek0", C.c_double), ("dEk", C.c_double), ("fi0", C.c_double), ("dfi", C.c_double),
        ("seo_Ek", d_p), ("seo_r", d_p), ("seo_pr", d_p), ("seo_perimeter", d_p),
    ]


class BunchDesc(C.Structure):
    _fields_ = [("n", C.c_int64), ("id0", C.c_int64), ("seed", C.c_uint64), ("sub_bunch", C.c_int64),
                ("transverse", C.c_int32), ("longitudinal", C.c_int32), ("cut_off", C.c_double),
                ("twiss", (C.c_double * 3) * 3), ("uniform_length", C.c_double), ("uniform_sigma", C.c_double),
                ("centre", C.c_double * 6), ("fi", C.c_double), ("bunch_id", C.c_double), ("out", C.c_void_p)]


DIST_TYPES = {"gauss": 0, "kv": 1, "waterbag": 2, "hollow_waterbag": 3, "UniformGauss": 4}


class SCDiag(C.Structure):
    _fields_ = [(name, C.c_double) for name in (
        "fi_s", "fi_e", "slice_step", "mean_gamma_m1", "mean_x", "mean_z", "sigma_x", "sigma_z",
        "xmin", "xmax", "zmin", "zmax", "dx", "dz", "bunch_length", "q_density")] + [
        ("count", C.c_int64), ("degenerate", C.c_int64)]


EXPORTS = {
    "ffa_bunch_sample": [C.POINTER(BunchDesc), d_p, d_p],
    "ffa_fieldmap_create": [C.POINTER(FieldDesc), d_p, C.POINTER(d_p)],
    "ffa_fieldmap_destroy": [d_p],
    "ffa_fieldmap_set_harmonics": [d_p, C.c_int32, d_p, d_p, d_p, d_p, d_p],
    "ffa_inject": [C.POINTER(StateSoA), C.c_int64, C.c_int64, d_p],
    "ffa_push": [d_p, C.POINTER(RFDesc), C.POINTER(Aperture), C.POINTER(Consts), C.POINTER(StepTable),
                 C.POINTER(StateSoA), C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                 d_p, d_p],
    "ffa_push_crossing": [d_p, C.POINTER(RFDesc), C.POINTER(Aperture), C.POINTER(Consts), C.POINTER(StepTable),
                          C.POINTER(StateSoA), C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                          d_p, d_p, C.POINTER(Crossing)],
    "ffa_aos_to_soa": [d_p, C.c_int64, C.POINTER(StateSoA), d_p],
    "ffa_mapgen": [C.POINTER(MapgenDesc), d_p],
    "ffa_theta_track": [d_p, C.POINTER(ThetaTrackDesc), d_p],
    "ffa_soa_to_aos": [C.POINTER(StateSoA), C.c_int64, d_p, d_p],
    "ffa_mean_fi": [C.POINTER(StateSoA), C.c_int64, d_p, d_p, d_p],
    "ffa_push_occupancy": [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
    "ffa_sc_plan_create": [C.POINTER(SCDesc), d_p, C.POINTER(d_p)],
    "ffa_sc_plan_destroy": [d_p],
    "ffa_sc_step": [d_p, C.POINTER(StateSoA), C.c_int64, C.c_int32, C.c_int32, d_p, d_p, d_p],
    "ffa_sc_buffers": [d_p, C.POINTER(d_p), C.POINTER(d_p), C.POINTER(d_p), C.POINTER(d_p),
                       C.POINTER(d_p), C.POINTER(d_p)],
    "ffa_sc_step_static": [C.POINTER(SCDesc), C.POINTER(StateSoA), C.c_int64, C.c_int32, C.c_int32, d_p, d_p, d_p],
    "ffa_mlp_train_step": [C.POINTER(MlpTrainDesc), d_p],
    "ffa_mlp_gemm": [d_p, C.c_int, C.c_int, d_p, C.c_int, C.c_int, d_p, C.c_int, C.c_int, C.c_int, C.c_int, d_p,
                     d_p],
    "ffa_mlp_gemm_timeouts": [C.POINTER(C.c_int32)],
    "ffa_mlp_pack": [d_p, d_p, d_p],
    "ffa_mlp_infer": [C.POINTER(MlpInferDesc), d_p],
}

SC_STATIC_MAX_PARTICLES = 524288
SC_STATIC_MAX_CELLS = 524288

_lib = None


def lib() -> C.CDLL:
    """The loaded libffa_cuda.so; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libffa_cuda.so not found at {LIB_PATH}: build it with `python -m pyffa_b200.build` "
                "(the tracking path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, argtypes in EXPORTS.items():
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = C.c_int
        _lib = L
    return _lib


class FFAError(RuntimeError):
    pass


def check(rc: int, what: str) -> None:
    if rc != FFA_OK:
        raise FFAError(f"{what} failed: {ERRORS.get(rc, rc)}")


def stream_ptr(stream) -> int:
    """cudaStream_t of a torch.cuda.Stream (0 = legacy default stream)."""
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(getattr(stream, "cuda_stream", stream))
