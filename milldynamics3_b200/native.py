"""Builds and loads the in-tree CUDA library (libmillgpu.so, sm_100a).

The library is the only compute path: there is no CPU fallback. `load()` raises when the shared
library is absent and cannot be built, and every C-ABI call fails with MG_ERR_NO_DEVICE when no
CUDA device is visible.
"""
from __future__ import annotations

import os
import subprocess

from . import capi

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libmillgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["mill_substeps_1024.cu", "mill_substeps_512.cu", "mill_kernels.cu", "mill_host.cu", "mill_params.cpp",
           "mill_noalloc.cu"]
# every header beside the sources (the build is stale when any of them is newer than the library)
HEADERS = sorted(f for f in os.listdir(os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc"))
                 if f.endswith((".cuh", ".h")))

# Arithmetic contract: IEEE f32 division and square root, no fused multiply-add contraction in
# device code (-fmad=false) or host code (-ffp-contract=off), no fast-math.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
              "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "millgpu.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles libmillgpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU): every
    source to an object in parallel, then one link."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    objs, procs = [], []
    for f in SOURCES:
        o = os.path.join(LIB_DIR, os.path.splitext(f)[0] + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", "-o", o, os.path.join(CSRC, f)]
        procs.append((cmd, subprocess.Popen(cmd, cwd=CSRC, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
        objs.append(o)
    logs, failed = [], []
    for cmd, p in procs:
        out, _ = p.communicate()
        logs.append(out)
        if p.returncode != 0:
            failed.append(" ".join(cmd) + "\n" + out)
    if failed:
        raise RuntimeError("building libmillgpu.so failed:\n" + "\n".join(failed))
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + objs
    r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("linking libmillgpu.so failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose:
        print("".join(logs) + r.stdout + r.stderr)
    for o in objs:
        os.remove(o)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_LIB = None


def load(build_if_missing: bool = True) -> capi.Lib:
    """Loads (building first if needed) the CUDA library; raises if it cannot be loaded."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if build_if_missing and _stale():
        build()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with milldynamics3_b200.native.build()")
    _LIB = capi.Lib(LIB_PATH, "mg_", capi.DEVICE_ONLY)
    return _LIB
