"""Builds libffa_cuda.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ with an ``extern "C"`` ABI (include/ffa_cuda.h);
Python reaches it through ctypes, so no torch extension is compiled.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_PATH = os.path.join(PKG_DIR, "libffa_cuda.so")
SOURCES = ["ffa_push.cu", "ffa_capi.cu", "ffa_sc.cu", "ffa_mapgen.cu", "ffa_mlp.cu", "ffa_bunch.cu"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc")
    if cand:
        return cand
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libffa_cuda.so")


def sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_rebuild() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(REPO_DIR, "include", "ffa_cuda.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu under csrc/ into pyffa_b200/libffa_cuda.so: one nvcc
    per source, run in parallel, then one link."""
    if not force and not needs_rebuild():
        return LIB_PATH
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    tmp = LIB_PATH + ".tmp"
    nvcc = nvcc_path()
    with tempfile.TemporaryDirectory(prefix="ffa_build_") as work:
        def compile_one(src):
            obj = os.path.join(work, os.path.basename(src) + ".o")
            cmd = [nvcc, *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-Xptxas", "-v" if verbose else "-O3", "-I", os.path.join(REPO_DIR, "include"),
                   "-c", src, "-o", obj]
            return obj, subprocess.run(cmd, capture_output=True, text=True)
        srcs = sources()
        with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
            results = list(ex.map(compile_one, srcs))
        for _, res in results:
            if res.returncode != 0:
                sys.stderr.write(res.stdout + res.stderr)
                raise RuntimeError("nvcc failed building libffa_cuda.so")
            if verbose:
                sys.stderr.write(res.stderr)
        res = subprocess.run([nvcc, *ARCH_FLAGS, "-shared", "-o", tmp, *[o for o, _ in results]],
                             capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("nvcc failed linking libffa_cuda.so")
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


PROBE_PATH = os.path.join(PKG_DIR, "libffa_probe.so")


def build_probe(force: bool = False) -> str:
    """The benchmark's FP64 peak probe (csrc/probe/ffa_probe.cu)."""
    src = os.path.join(CSRC, "probe", "ffa_probe.cu")
    if not force and os.path.exists(PROBE_PATH) and os.path.getmtime(PROBE_PATH) >= os.path.getmtime(src):
        return PROBE_PATH
    cmd = [nvcc_path(), *ARCH_FLAGS, "-O3", "-Xcompiler", "-fPIC", "-shared", "-o", PROBE_PATH, src]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libffa_probe.so")
    return PROBE_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
