"""Batches of independent mills in one launch per frame (the C ABI's mg_batch_*).

A batch is the unit of work of the reference's seed sweeps (`batch::run_seed`, batch.rs:40-191)
and parameter studies, run many mills at a time instead of one: every mill is an ordinary
`Simulation` (its own Params and seed) whose sub-steps run as one thread block of a shared
launch, so each mill's results are identical alone or in a batch.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import capi
from .sim import Backend, MillError, Simulation


class Batch:
    def __init__(self, backend: Backend, params_list):
        self.b = backend
        self.lib = backend.lib
        arr = (capi.Params * len(params_list))(*[p.copy() for p in params_list])
        h = C.c_void_p()
        rc = self.lib.batch_create(arr, len(params_list), C.byref(h))
        backend.check(rc)
        self.h = h
        self.params = [p.copy() for p in params_list]

    def __len__(self):
        return int(self.lib.batch_size(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        if rc != capi.MG_OK:
            m = self.lib.batch_last_error(self.h)
            raise MillError(rc, m.decode() if m else "")

    def set_options(self, cg_fp64: int = 0, block_threads: int = 0, sweep_warps: int = 0, spin_ns: int = 0,
                    block_regs: int = 0, sweep_order: int = 0):
        """Device options of every mill (MgOptions); block_regs = 64 runs the 64-register build,
        so that two blocks of 512 threads share an SM."""
        o = capi.Options()
        o.cg_fp64, o.block_threads, o.sweep_warps, o.spin_ns = cg_fp64, block_threads, sweep_warps, spin_ns
        o.block_regs = block_regs
        o.sweep_order = sweep_order
        self._c(self.lib.batch_set_options(self.h, C.byref(o)))

    def step_frames(self, frames: int = 1, frame_dt: float = 1.0 / 60.0):
        """Simulation::step(frame_dt) on every mill, `frames` times."""
        self._c(self.lib.batch_step_frames(self.h, frames, C.c_float(frame_dt)))

    def scalars(self):
        out = (capi.Scalars * len(self))()
        self._c(self.lib.batch_scalars(self.h, out))
        return list(out)

    def mill(self, i: int) -> Simulation:
        """A borrowed Simulation view of mill i (owned by the batch)."""
        h = C.c_void_p()
        self._c(self.lib.batch_mill(self.h, i, C.byref(h)))
        s = Simulation.__new__(Simulation)
        s.b, s.lib, s.h, s.params, s._owned, s._batch = self.b, self.lib, h, self.params[i].copy(), False, self
        return s

    def last_kernel_ms(self):
        ms = C.c_float()
        n = C.c_uint64()
        self._c(self.lib.batch_last_kernel_ms(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def stream(self) -> int:
        s = C.c_void_p()
        self._c(self.lib.batch_stream(self.h, C.byref(s)))
        return s.value or 0


def mix_params(backend: Backend, n: int, seed: int = 1, ball_diameter_m: float = 0.002):
    """A mix of n mills with the 512-mill batch's distributions: ball count log-uniform in
    [100, 3000] and ball fill J uniform in [0.2, 0.4] with the drum diameter that holds them,
    D = 2 r sqrt(N / (J phi)) (the reference derives the count from D and J, params.rs:558-566),
    redrawn until D lies in [40, 120] mm; fluid resolution uniform in [15, 60]; speed uniform in
    [50, 90] % of critical; each mill its own seed. Returns (params list, realised marginals)."""
    rng = np.random.default_rng(seed)
    base = backend.params_default()
    phi = float(base.media.packing_fraction_2d)
    r = 0.5 * ball_diameter_m
    out, info = [], []
    while len(out) < n:
        nb = math.exp(rng.uniform(math.log(100.0), math.log(3000.0)))
        j = rng.uniform(0.2, 0.4)
        d = 2.0 * r * math.sqrt(nb / (j * phi))
        if not (0.040 <= d <= 0.120):
            continue
        res = int(rng.integers(15, 61))
        speed = rng.uniform(50.0, 90.0)
        p = base.copy()
        p.mill.diameter_m = d
        p.mill.speed_mode = capi.SPEED_PERCENT_CRITICAL
        p.mill.speed_value = speed
        p.media.ball_diameter_m = ball_diameter_m
        p.media.fill_fraction = j
        p.simulation.resolution = res
        p.simulation.seed = seed * 100003 + len(out) + 1
        backend.validate(p)
        out.append(p)
        info.append({"diameter_m": d, "fill": j, "resolution": res, "speed_pct": speed})
    return out, info
