"""Python mirror of the reference's `Simulation` / `coupling::step_recorded` API over the C ABI.

Method names and argument meanings follow crates/mill-core/src/lib.rs (Simulation),
coupling.rs (step_recorded), pbf.rs (FluidParticles::step_coupled) and dem.rs
(DemState::step_recorded). Failures raise `MillError` carrying the library's message, the way the
reference returns `Err(String)` from `Simulation::new` / `set_params` (lib.rs:126-274).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi


class MillError(RuntimeError):
    """A non-OK status from the C ABI (invalid params, device error, capacity)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _f32(a, n2=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    return a


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(capi.f32p)


def unflatten_polygons(flat) -> list:
    """Inverse of flatten_polygons (surface.rs:420-430): [n_polys, len_0, x, y, ...] to a list of
    (len_k, 2) float32 arrays."""
    flat = np.asarray(flat, np.float32)
    polys, k = [], 1
    for _ in range(int(flat[0])):
        n = int(flat[k])
        polys.append(flat[k + 1:k + 1 + 2 * n].reshape(n, 2).copy())
        k += 1 + 2 * n
    if k != len(flat):
        raise ValueError(f"flattened polygons end at {k}, buffer holds {len(flat)}")
    return polys


@dataclass
class CouplingImpulses:
    """coupling.rs:37-63"""
    impulses: np.ndarray
    angular_impulses: np.ndarray
    clamp_hits: int
    fluid_momentum_change: np.ndarray


class Backend:
    """A bound library plus error plumbing."""

    def __init__(self, lib: capi.Lib):
        self.lib = lib

    def check(self, rc: int, handle=None):
        if rc != capi.MG_OK:
            msg = ""
            if handle is not None and hasattr(self.lib, "last_error"):
                m = self.lib.last_error(handle)
                msg = m.decode() if m else ""
            if not msg:
                m = self.lib.global_last_error()
                msg = m.decode() if m else ""
            raise MillError(rc, msg)

    # ---- params
    def params_default(self) -> capi.Params:
        p = capi.Params()
        self.check(self.lib.params_default(C.byref(p)))
        return p

    def validate(self, p: capi.Params):
        buf = C.create_string_buffer(512)
        rc = self.lib.params_validate(C.byref(p), buf, 512)
        if rc != capi.MG_OK:
            raise MillError(rc, buf.value.decode())

    def preset(self, p: capi.Params, pid: str) -> capi.Params:
        q = p.copy()
        self.check(self.lib.preset_apply(C.byref(q), pid.encode()))
        return q

    def derived(self, p: capi.Params) -> capi.Derived:
        d = capi.Derived()
        self.check(self.lib.params_derived(C.byref(p), C.byref(d)))
        return d


class Simulation:
    """lib.rs:82-566 `Simulation`, driving a handle of the bound library."""

    def __init__(self, backend: Backend, params: capi.Params, initial_balls=None):
        self.b = backend
        self.lib = backend.lib
        h = C.c_void_p()
        if initial_balls is None:
            rc = self.lib.sim_create(C.byref(params), C.byref(h))
        else:
            xy = _f32(initial_balls).reshape(-1)
            rc = self.lib.sim_create_with_balls(C.byref(params), _ptr(xy), len(xy) // 2, C.byref(h))
        self.b.check(rc)
        self.h = h
        self.params = params.copy()

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.lib.sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        self.b.check(rc, self.h)

    # ---- lib.rs
    def step(self, dt: float):
        self._c(self.lib.sim_step(self.h, C.c_float(dt)))

    def step_fixed(self):
        self._c(self.lib.sim_step_fixed(self.h))

    def reset_frame_stats(self):
        self._c(self.lib.sim_reset_frame_stats(self.h))

    def set_params(self, p: capi.Params):
        self._c(self.lib.sim_set_params(self.h, C.byref(p)))
        self.params = p.copy()

    def fixed_sub_dt(self) -> float:
        return float(self.lib.sim_fixed_sub_dt(self.h))

    def reset_energy_budget(self):
        self._c(self.lib.sim_reset_energy_budget(self.h))

    def set_options(self, cg_fp64: int = 0, block_threads: int = 0, sweep_warps: int = 0, spin_ns: int = 0,
                    mill_blocks: int = 0, test_wait_limit_us: int = 0, test_faults: int = 0, block_regs: int = 0,
                    sweep_order: int = 0):
        o = capi.Options()
        o.cg_fp64 = cg_fp64
        o.block_threads = block_threads
        o.sweep_warps = sweep_warps
        o.spin_ns = spin_ns
        o.mill_blocks = mill_blocks
        o.test_wait_limit_us = test_wait_limit_us
        o.test_faults = test_faults
        o.block_regs = block_regs
        o.sweep_order = sweep_order
        if hasattr(self.lib, "sim_set_options"):
            self._c(self.lib.sim_set_options(self.h, C.byref(o)))
        else:
            self._c(self.lib.sim_set_cg_fp64(self.h, cg_fp64))

    # ---- the path
    def coupling_step_recorded(self, drum: capi.Drum, drum_angle: float, media: capi.MediaParams,
                               slurry: capi.SlurryParams, dem_iterations: int, pbf_iterations: int, dt: float,
                               cap: int = 65536):
        fs, ds = capi.FluidStepStats(), capi.DemStepStats()
        recs = (capi.ImpactRecord * cap)()
        n = C.c_uint32()
        self._c(self.lib.coupling_step_recorded(self.h, C.byref(drum), C.c_float(drum_angle), C.byref(media),
                                                C.byref(slurry), dem_iterations, pbf_iterations, C.c_float(dt),
                                                C.byref(fs), C.byref(ds), recs, cap, C.byref(n)))
        return fs, ds, [recs[k] for k in range(min(n.value, cap))]

    def fluid_step_coupled(self, drum: capi.Drum, drum_angle: float, slurry: capi.SlurryParams, iterations: int,
                           dt: float):
        nb, _ = self.counts()
        fs = capi.FluidStepStats()
        imp = np.zeros(2 * max(nb, 1), np.float32)
        ang = np.zeros(max(nb, 1), np.float32)
        mom = np.zeros(2, np.float32)
        hits = C.c_uint32()
        self._c(self.lib.fluid_step_coupled(self.h, C.byref(drum), C.c_float(drum_angle), C.byref(slurry),
                                            iterations, C.c_float(dt), C.byref(fs), _ptr(imp), _ptr(ang),
                                            C.byref(hits), _ptr(mom)))
        return CouplingImpulses(imp[:2 * nb].reshape(-1, 2), ang[:nb], hits.value, mom), fs

    def dem_step(self, drum: capi.Drum, drum_angle: float, media: capi.MediaParams, iterations: int, dt: float,
                 external: CouplingImpulses | None = None, cap: int = 65536):
        ds = capi.DemStepStats()
        recs = (capi.ImpactRecord * cap)()
        n = C.c_uint32()
        imp = ang = None
        if external is not None:
            imp = _f32(external.impulses).reshape(-1)
            ang = _f32(external.angular_impulses).reshape(-1)
        self._c(self.lib.dem_step_recorded(self.h, C.byref(drum), C.c_float(drum_angle), C.byref(media), iterations,
                                           C.c_float(dt), _ptr(imp), _ptr(ang), C.byref(ds), recs, cap,
                                           C.byref(n)))
        return ds, [recs[k] for k in range(min(n.value, cap))]

    # ---- state
    def counts(self):
        nb, nf = C.c_uint32(), C.c_uint32()
        self._c(self.lib.get_counts(self.h, C.byref(nb), C.byref(nf)))
        return nb.value, nf.value

    def balls(self):
        nb, _ = self.counts()
        x = np.zeros(2 * max(nb, 1), np.float32)
        v = np.zeros(2 * max(nb, 1), np.float32)
        th = np.zeros(max(nb, 1), np.float32)
        om = np.zeros(max(nb, 1), np.float32)
        self._c(self.lib.get_balls(self.h, _ptr(x), _ptr(v), _ptr(th), _ptr(om)))
        return {"x": x[:2 * nb].reshape(-1, 2), "v": v[:2 * nb].reshape(-1, 2), "theta": th[:nb], "omega": om[:nb]}

    def set_balls(self, x, v=None, theta=None, omega=None):
        x = _f32(x).reshape(-1)
        n = len(x) // 2
        v = None if v is None else _f32(v).reshape(-1)
        theta = None if theta is None else _f32(theta).reshape(-1)
        omega = None if omega is None else _f32(omega).reshape(-1)
        self._c(self.lib.set_balls(self.h, n, _ptr(x), _ptr(v), _ptr(theta), _ptr(omega)))

    def ball_material(self) -> capi.BallMaterial:
        m = capi.BallMaterial()
        self._c(self.lib.get_ball_material(self.h, C.byref(m)))
        return m

    def set_ball_material(self, radius, mass, inertia, true_radius=None):
        m = capi.BallMaterial(radius, mass, inertia, radius if true_radius is None else true_radius)
        self._c(self.lib.set_ball_material(self.h, C.byref(m)))

    def fluid(self):
        _, nf = self.counts()
        x = np.zeros(2 * max(nf, 1), np.float32)
        v = np.zeros(2 * max(nf, 1), np.float32)
        dye = np.zeros(max(nf, 1), np.float32)
        g = np.zeros(2 * max(nf, 1), np.float32)
        gl = C.c_uint32()
        self._c(self.lib.get_fluid(self.h, _ptr(x), _ptr(v), _ptr(dye), _ptr(g), C.byref(gl)))
        return {"x": x[:2 * nf].reshape(-1, 2), "v": v[:2 * nf].reshape(-1, 2), "dye": dye[:nf],
                "viscous_guess": g[:2 * gl.value].reshape(-1, 2)}

    def set_fluid(self, x, v=None, dye=None, guess=None):
        x = _f32(x).reshape(-1)
        n = len(x) // 2
        v = None if v is None else _f32(v).reshape(-1)
        dye = None if dye is None else _f32(dye).reshape(-1)
        guess = None if guess is None else _f32(guess).reshape(-1)
        self._c(self.lib.set_fluid(self.h, n, _ptr(x), _ptr(v), _ptr(dye), _ptr(guess)))

    def fluid_material(self) -> capi.FluidMaterial:
        m = capi.FluidMaterial()
        self._c(self.lib.get_fluid_material(self.h, C.byref(m)))
        return m

    def set_fluid_material(self, particle_mass, h, rest_density):
        m = capi.FluidMaterial(particle_mass, h, rest_density)
        self._c(self.lib.set_fluid_material(self.h, C.byref(m)))

    # ---- outputs
    def scalars(self) -> capi.Scalars:
        s = capi.Scalars()
        self._c(self.lib.get_scalars(self.h, C.byref(s)))
        return s

    def energy_budget(self) -> capi.EnergyBudget:
        e = capi.EnergyBudget()
        self._c(self.lib.energy_budget(self.h, C.byref(e)))
        return e

    def state_hash(self, extended: bool = False) -> int:
        out = C.c_uint64()
        self._c(self.lib.state_hash(self.h, 1 if extended else 0, C.byref(out)))
        return out.value

    def mixing_index(self):
        m, valid = C.c_float(), C.c_int()
        self._c(self.lib.mixing_index(self.h, C.byref(m), C.byref(valid)))
        return m.value if valid.value else None

    def stress_histogram_rate(self):
        out = (C.c_double * capi.SE_BINS)()
        self._c(self.lib.stress_histogram_rate(self.h, out))
        return np.array(list(out))

    def metrics(self) -> capi.Metrics:
        """metrics::compute on the current state (metrics.rs:195-273)."""
        out = capi.Metrics()
        self._c(self.lib.metrics(self.h, C.byref(out)))
        return out

    def surface_flat(self) -> np.ndarray:
        """Simulation::fluid_surface flattened (lib.rs:354-361, surface.rs:233-272 and 420-430):
        [n_polys, len_0, x, y, ..., len_1, x, y, ...] as float32."""
        n = C.c_uint32(0)
        out = np.empty(capi.SURFACE_OUT_CAP, np.float32)
        self._c(self.lib.fluid_surface(self.h, _ptr(out), len(out), C.byref(n)))
        return out[:n.value].copy()

    def surface(self) -> list:
        """The free-surface polygons as a list of (n, 2) float32 arrays (surface.rs:233-272)."""
        return unflatten_polygons(self.surface_flat())

    def fluid_densities(self) -> np.ndarray:
        """FluidParticles::densities (pbf.rs:1124-1145) of the current positions."""
        out = np.zeros(max(self.counts()[1], 1), np.float32)
        self._c(self.lib.fluid_densities(self.h, _ptr(out)))
        return out[:self.counts()[1]]

    def surface_field(self):
        """build_field's masked occupancy field (MG_SURFACE_GRID^2 floats, row-major in gj) and
        analytic_phi_full (surface.rs:71-131)."""
        g = capi.SURFACE_GRID
        field = np.zeros((g, g), np.float32)
        phi = C.c_float(0.0)
        self._c(self.lib.surface_field(self.h, _ptr(field), C.byref(phi)))
        return field, phi.value

    def stress_metrics(self) -> capi.StressMetrics:
        """Simulation::metrics (lib.rs:383-390 over StressAccum::metrics, stress.rs:186-237)."""
        out = capi.StressMetrics()
        self._c(self.lib.stress_metrics(self.h, C.byref(out)))
        return out

    def last_step_stats(self):
        f, d, c = capi.FluidStepStats(), capi.DemStepStats(), capi.StepCounters()
        self._c(self.lib.last_step_stats(self.h, C.byref(f), C.byref(d), C.byref(c)))
        return f, d, c

    def last_neighbor_lists(self):
        _, nf = self.counts()
        off = np.zeros(nf + 1, np.uint32)
        ne = C.c_uint32()
        cap = 64 * max(nf, 1)
        nb = np.zeros(cap, np.uint32)
        self._c(self.lib.last_neighbor_lists(self.h, off.ctypes.data_as(capi.u32p), nb.ctypes.data_as(capi.u32p),
                                             cap, C.byref(ne)))
        return off, nb[:ne.value].copy()

    def last_ball_pairs(self):
        nbl, _ = self.counts()
        cap = 64 * max(nbl, 1)
        buf = np.zeros(2 * cap, np.uint32)
        n = C.c_uint32()
        self._c(self.lib.last_ball_pairs(self.h, buf.ctypes.data_as(capi.u32p), cap, C.byref(n)))
        return buf[:2 * n.value].reshape(-1, 2).copy()

    def drum(self) -> capi.Drum:
        d = self.b.derived(self.params)
        return capi.Drum(d.radius_m, d.omega, self.params.lifters)


def probe_grid(lib: capi.Lib, pts, cell: float):
    pts = _f32(pts).reshape(-1)
    n = len(pts) // 2
    mins = (C.c_int32 * 2)()
    wh = (C.c_int64 * 2)()
    cap = 2 * n + 1024
    cs = np.zeros(cap, np.uint32)
    idx = np.zeros(max(n, 1), np.uint32)
    nc = C.c_uint32()
    dense = C.c_int()
    rc = lib.probe_grid(_ptr(pts), n, C.c_float(cell), mins, wh, cs.ctypes.data_as(capi.u32p), cap,
                        idx.ctypes.data_as(capi.u32p), C.byref(nc), C.byref(dense))
    return rc, {"dense": dense.value, "min": (mins[0], mins[1]), "wh": (wh[0], wh[1]),
                "cell_start": cs[:nc.value].copy(), "indices": idx[:n].copy()}


def probe_candidate_pairs(lib: capi.Lib, pts, cell: float, cap: int | None = None):
    pts = _f32(pts).reshape(-1)
    n = len(pts) // 2
    cap = cap or max(64, 32 * n)
    buf = np.zeros(2 * cap, np.uint32)
    cnt = C.c_uint32()
    rc = lib.probe_candidate_pairs(_ptr(pts), n, C.c_float(cell), buf.ctypes.data_as(capi.u32p), cap, C.byref(cnt))
    return rc, buf[:2 * min(cnt.value, cap)].reshape(-1, 2).copy()


def probe_neighbor_lists(lib: capi.Lib, pts, h: float, cap: int | None = None):
    pts = _f32(pts).reshape(-1)
    n = len(pts) // 2
    cap = cap or max(64, 64 * n)
    off = np.zeros(n + 1, np.uint32)
    nb = np.zeros(cap, np.uint32)
    ne = C.c_uint32()
    rc = lib.probe_neighbor_lists(_ptr(pts), n, C.c_float(h), off.ctypes.data_as(capi.u32p),
                                  nb.ctypes.data_as(capi.u32p), cap, C.byref(ne))
    return rc, off, nb[:min(ne.value, cap)].copy()
