"""Errors of the f32 path against the FP64 oracle (the oracle's restatement built with
Real = double, oracle/liboracle64.so): per output after one sub-step from a common state, and
time-averaged statistics of multi-second runs over seeds.

Test infrastructure, like the oracle itself: the tests and the bench's CPU-baseline leg use it.
"""
from __future__ import annotations

import math
import os

import numpy as np

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Backend, Simulation

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE64_SO = os.path.join(ROOT, "oracle", "liboracle64.so")


def oracle64_backend(build=True):
    """The FP64 oracle behind the same C API as the parity oracle (built first unless `build` is
    false: the pool's worker processes only load what the parent built)."""
    from conftest import ORACLE_EXTRA, build_oracle
    if build:
        build_oracle()
    return Backend(capi.Lib(ORACLE64_SO, "or_", ORACLE_EXTRA))


def copy_state(src: Simulation, dst: Simulation):
    """Gives dst exactly src's f32 state (balls, fluid, materials, viscous warm start)."""
    bl = src.balls()
    dst.set_balls(bl["x"], bl["v"], bl["theta"], bl["omega"])
    bm = src.ball_material()
    dst.set_ball_material(bm.radius, bm.mass, bm.inertia, bm.true_radius)
    fl = src.fluid()
    g = fl["viscous_guess"]
    dst.set_fluid(fl["x"], fl["v"], fl["dye"], g if len(g) == len(fl["x"]) and len(g) else None)
    fm = src.fluid_material()
    dst.set_fluid_material(fm.particle_mass, fm.h, fm.rest_density)


def _rel(a, ref):
    """Norm-wise relative error |a - ref| / |ref| over the array (and the largest absolute one)."""
    a = np.asarray(a, np.float64).reshape(-1)
    ref = np.asarray(ref, np.float64).reshape(-1)
    if a.size == 0:
        return {"rel": 0.0, "max_abs": 0.0}
    d = a - ref
    den = float(np.linalg.norm(ref))
    return {"rel": float(np.linalg.norm(d)) / den if den > 0 else float(np.linalg.norm(d)),
            "max_abs": float(np.abs(d).max())}


OUTPUTS = ("ball_x", "ball_v", "ball_omega", "ball_theta", "fluid_x", "fluid_v", "fluid_wall_work_j",
           "dem_wall_work_j", "dem_dissipated_energy_j", "fluid_ke_delta_viscosity_j", "mean_shear_rate_per_s")


def _outputs(s: Simulation):
    bl, fl = s.balls(), s.fluid()
    fs, ds, _ = s.last_step_stats()
    return {"ball_x": bl["x"], "ball_v": bl["v"], "ball_omega": bl["omega"], "ball_theta": bl["theta"],
            "fluid_x": fl["x"], "fluid_v": fl["v"], "fluid_wall_work_j": fs.wall_work_j,
            "dem_wall_work_j": ds.wall_work_j, "dem_dissipated_energy_j": ds.dissipated_energy_j,
            "fluid_ke_delta_viscosity_j": fs.ke_delta_viscosity_j,
            "mean_shear_rate_per_s": fs.mean_shear_rate_per_s}


def single_step_errors(f32_backends, f64: Backend, params, warm_frames=30, cg_fp64=(0,)):
    """Steps the mill `params` for warm_frames frames on the first f32 backend, hands that state to
    every backend (the f32 ones and the FP64 oracle) and runs one coupled sub-step on each.
    Returns {label: {output: {rel, max_abs}}} of each f32 run against the FP64 oracle, labels
    '<backend index>/cg_fp64=<mode>'."""
    base = Simulation(f32_backends[0], params)
    for _ in range(warm_frames):
        base.step(1.0 / 60.0)
    ref = Simulation(f64, params)
    copy_state(base, ref)
    ref.step_fixed()
    want = _outputs(ref)
    out = {}
    for k, b in enumerate(f32_backends):
        for mode in cg_fp64:
            s = Simulation(b, params)
            copy_state(base, s)
            s.set_options(cg_fp64=mode)
            s.step_fixed()
            got = _outputs(s)
            out["%d/cg_fp64=%d" % (k, mode)] = {o: _rel(got[o], want[o]) for o in OUTPUTS}
            s.close()
    base.close()
    ref.close()
    return out


STAT_NAMES = ("power_draw_w", "torque_nm", "mixing_index", "impact_rate_per_s")


def run_statistics(b: Backend, params, settle_s, measure_s, init_from=None):
    """Time averages of one run over the measured window: power draw, torque and mixing index (the
    per-frame readings averaged over frames; power and torque are lib.rs's EMA readings) and the
    summed rate of the 28-bin impact-energy histogram at the end (stress.rs's EMA rates).
    init_from: a Simulation whose initial state the run starts from."""
    s = Simulation(b, params)
    if init_from is not None:
        copy_state(init_from, s)
    return _window(s, settle_s, measure_s)


def _window(s: Simulation, settle_s, measure_s):
    for _ in range(int(round(settle_s * 60))):
        s.step(1.0 / 60.0)
    p = t = mi = 0.0
    n = int(round(measure_s * 60))
    for _ in range(n):
        s.step(1.0 / 60.0)
        sc = s.scalars()
        p += sc.power_draw_w
        t += sc.torque_nm
        m = s.mixing_index()
        mi += m if m is not None else math.nan
    hist = float(np.sum(s.stress_histogram_rate()))
    s.close()
    return {"power_draw_w": p / n, "torque_nm": t / n, "mixing_index": mi / n, "impact_rate_per_s": hist}


def _seed_params(b, params, seed):
    p = params.copy()
    p.simulation.seed = seed
    return p


def ensemble_gate(f32: Backend, f64: Backend, params, seeds, settle_s, measure_s, pool=None):
    """The multi-second acceptance gate: for every seed the f32 run and the FP64-oracle run from the
    same initial state (the f32 seeding); returns ({stat: (f32 mean over seeds, FP64 mean, relative
    difference)}, per-seed f32 values, per-seed FP64 values). With a process pool the FP64 runs go
    to it first and the f32 runs proceed meanwhile."""
    jobs = []
    for seed in seeds:
        p = _seed_params(f32, params, seed)
        init = Simulation(f32, p)
        bm, fm = init.ball_material(), init.fluid_material()
        st = (init.balls(), (bm.radius, bm.mass, bm.inertia, bm.true_radius), init.fluid(),
              (fm.particle_mass, fm.h, fm.rest_density))
        init.close()
        jobs.append((p, st))
    args = [(bytes(p), st, settle_s, measure_s) for p, st in jobs]
    pending = pool.map_async(_fp64_job, args) if pool is not None else None
    a = [run_statistics(f32, p, settle_s, measure_s) for p, _ in jobs]
    r = pending.get() if pending is not None else [_fp64_job(x, f64) for x in args]
    out = {}
    for k in STAT_NAMES:
        ma = float(np.mean([x[k] for x in a]))
        mr = float(np.mean([x[k] for x in r]))
        out[k] = (ma, mr, abs(ma - mr) / abs(mr) if mr != 0 else math.inf)
    return out, a, r


def _fp64_job(job, f64=None):
    """One FP64-oracle run (picklable for a process pool): params bytes, the f32 initial state."""
    pbytes, (bl, bm, fl, fm), settle_s, measure_s = job
    if f64 is None:
        f64 = oracle64_backend(build=False)
    p = capi.Params.from_buffer_copy(pbytes)
    s = Simulation(f64, p)
    s.set_balls(bl["x"], bl["v"], bl["theta"], bl["omega"])
    s.set_ball_material(*bm)
    s.set_fluid(fl["x"], fl["v"], fl["dye"], None)
    s.set_fluid_material(*fm)
    return _window(s, settle_s, measure_s)
