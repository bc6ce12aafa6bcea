"""Shared fixtures: the oracle (CPU restatement, the checker) and the device library (CUDA)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from milldynamics3_b200 import capi  # noqa: E402
from milldynamics3_b200.sim import Backend  # noqa: E402

ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
ORACLE64_SO = os.path.join(ORACLE_DIR, "liboracle64.so")  # the same restatement in f64

P = C.POINTER
ORACLE_EXTRA = [
    ("sim_set_cg_fp64", C.c_int, [C.c_void_p, C.c_int]),
    ("stress_set_debounce_factor", C.c_int, [C.c_void_p, C.c_double]),
    ("total_mechanical_energy", C.c_double, [C.c_void_p]),
    ("probe_near", C.c_int, [capi.f32p, C.c_uint32, C.c_float, C.c_float, C.c_float, capi.u32p, C.c_uint32,
                             capi.u32p]),
    ("sdf_world", None, [P(capi.Drum), C.c_float, C.c_float, C.c_float, capi.f32p, capi.f32p, capi.f32p]),
    ("sdf_local", C.c_float, [P(capi.Drum), C.c_float, C.c_float]),
    ("toi_swept", C.c_int, [P(capi.Drum), C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                            C.c_float, capi.f32p]),
    ("effective_friction", C.c_float, [C.c_float, C.c_float, C.c_float, C.c_float]),
    ("impact_energy_bin", C.c_int, [C.c_float]),
    ("rng_next_u64", C.c_uint64, [P(C.c_uint64)]),
    ("rng_seed_state", C.c_uint64, [C.c_uint64]),
    ("rng_next_f32", C.c_float, [P(C.c_uint64)]),
    ("se_bin", C.c_int, [C.c_double]),
]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: multi-second simulations")


def build_oracle():
    srcs = [f for f in os.listdir(ORACLE_DIR) if f.endswith((".cpp", ".hpp"))] + ["Makefile"]
    newest = max(os.path.getmtime(os.path.join(ORACLE_DIR, f)) for f in srcs)
    newest = max(newest, os.path.getmtime(os.path.join(ROOT, "include", "millgpu.h")))
    stale = [so for so in (ORACLE_SO, ORACLE64_SO) if not os.path.exists(so) or os.path.getmtime(so) < newest]
    if stale:
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "all"], check=True)
    return ORACLE_SO


@pytest.fixture(scope="session")
def oracle_lib():
    return capi.Lib(build_oracle(), "or_", ORACLE_EXTRA)


@pytest.fixture(scope="session")
def oracle64():
    build_oracle()
    return Backend(capi.Lib(ORACLE64_SO, "or_", ORACLE_EXTRA))


@pytest.fixture(scope="session")
def oracle(oracle_lib):
    return Backend(oracle_lib)


@pytest.fixture(scope="session")
def device_lib():
    from milldynamics3_b200 import native
    return native.load()


@pytest.fixture(scope="session")
def device(device_lib):
    return Backend(device_lib)
