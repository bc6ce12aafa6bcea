"""Seed sweeps: the reference's `batch::run_seed` and `batch::combine` (batch.rs:40-191).

`run_seeds` runs one Params under several seeds for `warmup_revolutions`, then averages the
stress metrics frame by frame over `measure_revolutions`. On the device library every seed is a
mill of one batch, so a frame of the whole sweep is one launch; each seed's numbers are those of
`run_seed` for that seed alone (the oracle computes them one seed after the other).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .sim import Backend, MillError


def value_names(backend: Backend):
    """The 23 scalar names of a SeedResult, in order (batch.rs:109-139)."""
    return [backend.lib.seed_value_name(k).decode() for k in range(capi.SEED_VALUES)]


@dataclass
class SeedResult:
    seed: int
    window_s: float
    coarse_graining_factor: float
    names: list
    values: list
    power_drift_rel_per_rev: float

    def get(self, name: str) -> float:
        return self.values[self.names.index(name)]


@dataclass
class Combined:
    names: list
    mean: list
    std_err: list
    seeds: int


def _check(backend: Backend, rc: int):
    if rc != capi.MG_OK:
        m = backend.lib.global_last_error()
        raise MillError(rc, m.decode() if m else "")


def run_seeds(backend: Backend, params: capi.Params, seeds, warmup_revolutions: float,
              measure_revolutions: float):
    """run_seed (batch.rs:40-107) for every seed; returns one SeedResult per seed."""
    seeds = [int(s) for s in seeds]
    arr = (C.c_uint64 * len(seeds))(*seeds)
    out = (capi.SeedResult * max(len(seeds), 1))()
    _check(backend, backend.lib.seed_sweep(C.byref(params), arr, len(seeds), C.c_float(warmup_revolutions),
                                           C.c_float(measure_revolutions), out))
    names = value_names(backend)
    return [SeedResult(r.seed, r.window_s, r.coarse_graining_factor, names, list(r.values),
                       r.power_drift_rel_per_rev) for r in out[:len(seeds)]]


def run_seed(backend: Backend, params: capi.Params, seed: int, warmup_revolutions: float,
             measure_revolutions: float) -> SeedResult:
    return run_seeds(backend, params, [seed], warmup_revolutions, measure_revolutions)[0]


def combine(backend: Backend, results) -> Combined:
    """Mean and standard error (n - 1) of every scalar over seeds (batch.rs:161-191)."""
    if not results:
        raise MillError(capi.MG_ERR_ARG, "no results to combine")
    if any(r.names != results[0].names for r in results):
        raise MillError(capi.MG_ERR_ARG, "results have different scalar names")
    arr = (capi.SeedResult * len(results))()
    for a, r in zip(arr, results):
        a.seed, a.window_s, a.coarse_graining_factor = r.seed, r.window_s, r.coarse_graining_factor
        a.power_drift_rel_per_rev = r.power_drift_rel_per_rev
        for k, v in enumerate(r.values):
            a.values[k] = v
    mean = (C.c_double * capi.SEED_VALUES)()
    se = (C.c_double * capi.SEED_VALUES)()
    _check(backend, backend.lib.seed_combine(arr, len(results), mean, se))
    return Combined(list(results[0].names), list(mean), list(se), len(results))


def drift_per_rev(backend: Backend, y, frames_per_rev: float) -> float:
    """Least-squares slope of y relative to its mean, per revolution (batch.rs:141-159)."""
    a = np.ascontiguousarray(y, dtype=np.float64)
    return float(backend.lib.seed_drift_per_rev(a.ctypes.data_as(C.POINTER(C.c_double)), len(a),
                                                 C.c_double(frames_per_rev)))
