"""The C-ABI library: it builds for sm_100a, loads without a GPU, and
exports every entry point include/ffa_cuda.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

from pyffa_b200 import _lib, build

HEADER = os.path.join(build.REPO_DIR, "include", "ffa_cuda.h")


def declared_entry_points():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(ffa_\w+)\s*\(", text)))


def test_library_builds_and_exports_header_symbols():
    path = build.build()
    assert os.path.exists(path)
    L = ctypes.CDLL(path)
    names = declared_entry_points()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_entry_points()) == set(_lib.EXPORTS)


def test_struct_sizes_match_header():
    # sizes of the ABI structs as the C compiler lays them out
    import subprocess
    import tempfile
    src = r'''
#include <stdio.h>
#include "ffa_cuda.h"
int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %d %d %d %d %d %d\n", sizeof(ffa_field_desc),
 sizeof(ffa_rf_desc), sizeof(ffa_aperture), sizeof(ffa_consts), sizeof(ffa_state_soa), sizeof(ffa_step_table),
 sizeof(ffa_sc_desc), sizeof(ffa_sc_diag), sizeof(ffa_crossing), sizeof(ffa_mapgen_desc), sizeof(ffa_theta_track_desc),
 sizeof(ffa_mlp_train_desc), sizeof(ffa_mlp_infer_desc), sizeof(void*), FFA_CROSSING_RECORD, FFA_MLP_HIDDEN,
 FFA_MLP_PARAMS, FFA_MLP_WPACK_BYTES, FFA_MLP_SPLIT_WORK, FFA_FIT_SUMS); return 0;}
'''
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "s.c"), "w") as f:
        f.write(src)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I", os.path.dirname(HEADER), "-o", os.path.join(d, "s"), os.path.join(d, "s.c")], check=True)
    out = subprocess.run([os.path.join(d, "s")], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(x) for x in out]
    py = [ctypes.sizeof(t) for t in (_lib.FieldDesc, _lib.RFDesc, _lib.Aperture, _lib.Consts, _lib.StateSoA,
                                     _lib.StepTable, _lib.SCDesc, _lib.SCDiag, _lib.Crossing,
                                     _lib.MapgenDesc, _lib.ThetaTrackDesc, _lib.MlpTrainDesc, _lib.MlpInferDesc)] + \
        [ctypes.sizeof(ctypes.c_void_p), _lib.CROSSING_RECORD, _lib.MLP_HIDDEN, _lib.MLP_PARAMS, _lib.MLP_WPACK_BYTES,
                                               _lib.MLP_SPLIT_WORK, _lib.FIT_SUMS]
    assert sizes == py


def test_invalid_arguments_rejected_without_gpu():
    L = _lib.lib()
    # argument validation happens before any CUDA call
    assert L.ffa_fieldmap_create(None, None, None) == 1
    out = ctypes.c_void_p()
    d = _lib.FieldDesc()
    d.nsectors = 0
    assert L.ffa_fieldmap_create(ctypes.byref(d), None, ctypes.byref(out)) == 1
    d.nsectors = 12
    d.max_order = 9
    assert L.ffa_fieldmap_create(ctypes.byref(d), None, ctypes.byref(out)) == 4
    assert L.ffa_push(None, None, None, None, None, None, 0, 0, 0, 0.0, 0, 0, None, None) == 1
    assert L.ffa_fieldmap_set_harmonics(None, 0, None, None, None, None, None) == 1
    assert L.ffa_aos_to_soa(None, 0, None, None) == 1
    # learned sector map entry points
    assert L.ffa_mlp_train_step(None, None) == 1
    assert L.ffa_mlp_gemm(None, 1, 0, None, 1, 0, None, 1, 1, 1, 1, None, None) == 1
    assert L.ffa_mlp_pack(None, None, None) == 1
    assert L.ffa_mlp_infer(None, None) == 1
    t = _lib.MlpTrainDesc()
    t.batch = 16
    t.n_fit = 9
    assert L.ffa_mlp_train_step(ctypes.byref(t), None) == 1


def test_train_schedule_fields_checked_without_gpu():
    """The device schedule needs both lr_table and counter; the host
    schedule needs step >= 1 when it updates (checked before any launch)."""
    L = _lib.lib()
    keep = ctypes.create_string_buffer(64)
    fake = ctypes.addressof(keep)
    t = _lib.MlpTrainDesc()
    t.batch, t.n_fit = 16, 4
    for name in ("params", "grads", "adam_m", "adam_v", "x", "target", "work", "loss_part"):
        setattr(t, name, fake)
    t.lr_table = fake                      # counter missing
    assert L.ffa_mlp_train_step(ctypes.byref(t), None) == 1
    t.lr_table, t.counter = None, fake     # lr_table missing
    assert L.ffa_mlp_train_step(ctypes.byref(t), None) == 1
    t.counter = None
    t.lr, t.step = 1e-3, 0                 # host schedule, update without a step number
    assert L.ffa_mlp_train_step(ctypes.byref(t), None) == 1
    assert L.ffa_mlp_gemm_timeouts(None) == 1


def test_soa_offset_advances_each_column_by_its_element_size():
    st = _lib.StateSoA()
    base = 1 << 20
    for k, (name, _) in enumerate(_lib.StateSoA._fields_):
        if name not in ("sc_pp", "e_pp_fi"):           # two columns left null
            setattr(st, name, base + (k << 16))
    out = _lib.soa_offset(st, 10)
    sizes = {"inj": 1, "surv": 1, "sc_pre": 1, "sc_pp": 1, "inj_step": 4}
    for k, (name, _) in enumerate(_lib.StateSoA._fields_):
        if name in ("sc_pp", "e_pp_fi", "order"):   # the thread order is a permutation of the whole range
            assert getattr(out, name) is None
        else:
            assert getattr(out, name) == base + (k << 16) + 10 * sizes.get(name, 8), name
    # the header's column types: uint8 flags, int32 injection steps, double otherwise
    text = open(HEADER).read()
    assert "uint8_t *inj, *surv;" in text and "const int32_t *inj_step;" in text and "uint8_t *sc_pre, *sc_pp;" in text


def test_every_entry_point_cites_what_it_replaces():
    """Each declaration's doc block (the last comment starting at column 0
    before it) cites the reference file it replaces or says that it has no
    counterpart there."""
    text = open(HEADER).read()
    bad = []
    for m in re.finditer(r"\bint\s+(ffa_\w+)\s*\(", text):
        before = text[:m.start()]
        if before.rfind("/*") > before.rfind("*/"):
            continue                      # a mention inside a comment
        start = before.rfind("\n/*")
        doc = before[start:before.find("*/", start)]
        if not any(key in doc for key in ("src/", "examples/", "benchmarks/", "counterpart")):
            bad.append(m.group(1))
    assert not bad, bad


def test_empty_bunch_accepted_without_columns():
    """n = 0 with every column NULL: the conversions and the injection
    return 0 without touching the device (argument checks come first)."""
    st = _lib.StateSoA()
    L = _lib.lib()
    assert L.ffa_aos_to_soa(None, 0, ctypes.byref(st), None) == 0
    assert L.ffa_soa_to_aos(ctypes.byref(st), 0, None, None) == 0
    assert L.ffa_inject(ctypes.byref(st), 0, 0, None) == 0
    assert L.ffa_aos_to_soa(None, 1, ctypes.byref(st), None) == 1      # a particle needs its columns
