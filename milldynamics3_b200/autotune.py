"""Autotuner of the launch shapes: for a mill (or a batch of mills) it times the candidate device
options on the device itself and keeps the fastest, after checking that every candidate leaves
the same state bits (the options change how the work is spread over threads and blocks, never
the arithmetic, so a candidate that changed a result would be a defect, not a trade-off).

Single mill (mg_sim_* handles): the mill's block size and register budget (1,024 threads at 64
registers, 512 at 128), the number of blocks sharing its per-ball stages (mill_blocks) and the
warps taking balls in the drag and buoyancy sweeps (sweep_warps). Batches (mg_batch_*): the block
size and register budget of the one-block-per-mill launch (1,024 threads, 512 at 128 registers
with one block per SM, or 512 at 64 registers with two blocks per SM).

Choices are remembered per size bucket, (fluid particles, balls) rounded to powers of two, in a
JSON table that can be saved and loaded, so a serving process tunes each bucket once.
"""
from __future__ import annotations

import json
import math
import time
from dataclasses import asdict, dataclass, field

from . import capi
from .sim import Backend, Simulation

MILL_CANDIDATES = [
    {"block_threads": 1024, "mill_blocks": 16, "sweep_warps": 32},
    {"block_threads": 1024, "mill_blocks": 8, "sweep_warps": 32},
    {"block_threads": 1024, "mill_blocks": 16, "sweep_warps": 16},
    {"block_threads": 1024, "mill_blocks": 4, "sweep_warps": 32},
    {"block_threads": 1024, "mill_blocks": 1, "sweep_warps": 32},
    {"block_threads": 512, "mill_blocks": 16, "sweep_warps": 16},
]
BATCH_CANDIDATES = [
    {"block_threads": 1024, "block_regs": 0},
    {"block_threads": 512, "block_regs": 0},
    {"block_threads": 512, "block_regs": 64},
]


def bucket(nf: int, nb: int) -> str:
    """The size bucket of a mill: fluid particles and balls, each rounded up to a power of two."""
    up = lambda n: 0 if n <= 0 else 1 << int(math.ceil(math.log2(n)))
    return "nf%d_nb%d" % (up(nf), up(nb))


@dataclass
class Tuned:
    options: dict
    ms: float
    timings: dict = field(default_factory=dict)


class Autotuner:
    def __init__(self, backend: Backend, frames: int = 3):
        self.b = backend
        self.frames = frames
        self.table: dict[str, dict] = {}

    # ---- persistence
    def save(self, path: str):
        with open(path, "w") as f:
            json.dump(self.table, f, indent=1, sort_keys=True)

    def load(self, path: str):
        with open(path) as f:
            self.table.update(json.load(f))

    # ---- single mills
    def _time_mill(self, params, balls, opts):
        s = Simulation(self.b, params, initial_balls=balls)
        s.set_options(**opts)
        s.step(1.0 / 60.0)  # warm-up frame (first launch, allocations)
        t0 = time.perf_counter()
        for _ in range(self.frames):
            s.step(1.0 / 60.0)
        dt = (time.perf_counter() - t0) / self.frames
        h = s.state_hash(True)
        s.close()
        return dt, h

    def tune_mill(self, params, balls=None, candidates=None) -> Tuned:
        """Times every candidate on this mill (a warm-up frame, then `frames` frames each, the
        state hashes compared) and records the fastest for the mill's size bucket."""
        probe = Simulation(self.b, params, initial_balls=balls)
        nb, nf = probe.counts()
        probe.close()
        times, hashes = {}, {}
        for opts in candidates or MILL_CANDIDATES:
            key = json.dumps(opts, sort_keys=True)
            times[key], hashes[key] = self._time_mill(params, balls, opts)
        if len(set(hashes.values())) != 1:
            raise RuntimeError("launch options changed the results: %s" % hashes)
        best = min(times, key=times.get)
        t = Tuned(json.loads(best), 1e3 * times[best], {k: 1e3 * v for k, v in times.items()})
        self.table[bucket(nf, nb)] = asdict(t)
        return t

    def mill_options(self, params, balls=None) -> dict:
        """The tuned options of the mill's bucket (tuning it first when it has no entry)."""
        probe = Simulation(self.b, params, initial_balls=balls)
        nb, nf = probe.counts()
        probe.close()
        key = bucket(nf, nb)
        if key not in self.table:
            self.tune_mill(params, balls)
        return dict(self.table[key]["options"])

    # ---- batches
    def tune_batch(self, params_list, candidates=None) -> Tuned:
        """Times every batch candidate on this mix (a warm-up frame, then `frames` frames each, every
        mill's state hash compared) and records the fastest under the key 'batch'."""
        from .batch import Batch
        times, hashes = {}, {}
        for opts in candidates or BATCH_CANDIDATES:
            key = json.dumps(opts, sort_keys=True)
            bt = Batch(self.b, params_list)
            bt.set_options(**opts)
            bt.step_frames(1)
            t0 = time.perf_counter()
            bt.step_frames(self.frames)
            times[key] = (time.perf_counter() - t0) / self.frames
            hashes[key] = tuple(bt.mill(i).state_hash(True) for i in range(len(params_list)))
            bt.close()
        if len(set(hashes.values())) != 1:
            raise RuntimeError("launch options changed the results of a batch")
        best = min(times, key=times.get)
        t = Tuned(json.loads(best), 1e3 * times[best], {k: 1e3 * v for k, v in times.items()})
        self.table["batch"] = asdict(t)
        return t


def apply_mill_options(sim: Simulation, opts: dict):
    sim.set_options(**opts)


def options_struct(opts: dict) -> capi.Options:
    o = capi.Options()
    for k, v in opts.items():
        setattr(o, k, v)
    return o
