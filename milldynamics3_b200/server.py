"""Request server of mill jobs with continuous batching (the C ABI's mg_server_*).

Jobs (Params plus a simulated horizon) are queued, admitted oldest first whenever the device
bytes of their state fit under the budget, advanced together one frame per step (one launch for
all running jobs) and retired at their horizon; every step streams back each running job's
power, torque and impact-energy histogram. A job's results are identical to the same mill
stepped alone, whatever else is in the mix.
"""
from __future__ import annotations

import ctypes as C

from . import capi
from .sim import Backend, MillError


class Server:
    def __init__(self, backend: Backend, memory_budget_bytes: int = 0, max_active: int = 0,
                 block_threads: int = 0, frame_dt: float = 1.0 / 60.0):
        self.b = backend
        self.lib = backend.lib
        cfg = capi.ServerConfig()
        cfg.memory_budget_bytes = memory_budget_bytes
        cfg.max_active = max_active
        cfg.block_threads = block_threads
        cfg.frame_dt = frame_dt
        h = C.c_void_p()
        backend.check(self.lib.server_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        if rc != capi.MG_OK:
            m = self.lib.server_last_error(self.h)
            raise MillError(rc, m.decode() if m else "")

    def submit(self, params: capi.Params, horizon_s: float) -> int:
        jid = C.c_uint64()
        self._c(self.lib.server_submit(self.h, C.byref(params), C.c_double(horizon_s), C.byref(jid)))
        return jid.value

    def submit_sweep(self, params: capi.Params, n_seeds: int, warmup_revolutions: float,
                     measure_revolutions: float) -> int:
        """A seed-sweep job: seeds 1..n_seeds of `params`, each batch::run_seed over the window,
        sharing the server's launches with the other jobs (web/src/batch/plan.ts semantics).
        Returns the sweep id (cancel() takes it too)."""
        sid = C.c_uint64()
        self._c(self.lib.server_submit_sweep(self.h, C.byref(params), n_seeds, C.c_float(warmup_revolutions),
                                             C.c_float(measure_revolutions), C.byref(sid)))
        return sid.value

    def sweep_result(self, sweep_id: int, n_seeds: int):
        """(state, seeds finished, per-seed SeedResults, mean, std_err); the last three are None
        until the sweep has FINISHED."""
        res = (capi.SeedResult * n_seeds)()
        mean = (C.c_double * capi.SEED_VALUES)()
        se = (C.c_double * capi.SEED_VALUES)()
        st, done = C.c_uint32(), C.c_uint32()
        self._c(self.lib.server_sweep_result(self.h, C.c_uint64(sweep_id), res, mean, se, C.byref(st),
                                             C.byref(done)))
        if st.value != capi.JOB_FINISHED:
            return st.value, done.value, None, None, None
        return st.value, done.value, [r.copy() for r in res], list(mean), list(se)

    def release_sweep(self, sweep_id: int):
        """Forgets the sweep's record (its result cannot be read afterwards); seeds still queued
        or running are cancelled."""
        self._c(self.lib.server_sweep_release(self.h, C.c_uint64(sweep_id)))

    def cancel(self, job_id: int):
        self._c(self.lib.server_cancel(self.h, C.c_uint64(job_id)))

    def step(self):
        """Admits what fits, advances every running job by one frame, retires the finished."""
        self._c(self.lib.server_step(self.h))

    def poll(self, cap: int = 4096):
        """Pending updates (oldest first), as capi.JobUpdate copies."""
        out = []
        buf = (capi.JobUpdate * cap)()
        while True:
            n = C.c_uint32()
            self._c(self.lib.server_poll(self.h, buf, cap, C.byref(n)))
            out.extend(buf[k].copy() for k in range(n.value))
            if n.value < cap:
                return out

    def stats(self) -> capi.ServerStats:
        s = capi.ServerStats()
        self._c(self.lib.server_stats(self.h, C.byref(s)))
        return s
