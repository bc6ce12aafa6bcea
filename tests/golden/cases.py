"""Scenario definitions shared by the fixture generator (make_golden.py) and the tests that
check the oracle and the device against the committed fixtures (oracle_states.json).

Each case is a mill built through the C ABI's Params (the reference's Params::default() plus
overrides, params.rs:62-77 and following) and advanced by Simulation::step / step_fixed
(lib.rs:438-464). The workloads follow the configurations the benchmark is quoted on:
  * realtime: the 'realtime' preset exactly as Params supplies it (63 mm drum, 407 discs,
    794 fluid particles, 24 sub-steps per frame);
  * realtime_300: the same mill with 300 steel discs (7800 kg/m^3) placed uniformly at random
    without overlap in the lower drum (Simulation::with_initial_balls, lib.rs:138-204). The lower
    half alone would need a packing of 0.65, past what random placement reaches (~0.55), so the
    discs fill the part of the drum below 0.35 R (packing 0.45);
  * dem_500: balls only (slurry off): 500 discs of 10 mm, 7800 kg/m^3, friction 0.3, restitution
    0.5, 30 % fill, 60 % of critical speed, in a 0.45 m drum (the 1 m drum of the large-N case
    scaled to hold 500 discs of 5 mm radius);
  * large_res100: 5,000 discs of 2 mm in a 221 mm drum with fluid resolution 100 (~12.7k fluid
    particles), viscosity 1e-3 and 1e-1 Pa s.
"""
from __future__ import annotations

import math

import numpy as np


def set_path(p, path, value):
    obj = p
    parts = path.split(".")
    for part in parts[:-1]:
        obj = getattr(obj, part)
    setattr(obj, parts[-1], value)


def dem_500(p):
    from milldynamics3_b200 import capi
    for k, v in {"slurry.enabled": 0, "mill.diameter_m": 0.45, "mill.speed_mode": capi.SPEED_PERCENT_CRITICAL,
                 "mill.speed_value": 60.0, "media.fill_fraction": 0.3, "media.ball_diameter_m": 0.01,
                 "media.density_kg_m3": 7800.0, "media.friction_ball_ball": 0.3, "media.friction_ball_wall": 0.3,
                 "media.friction_ball_ball_static": 0.3, "media.friction_ball_wall_static": 0.3,
                 "media.restitution_ball_ball": 0.5, "media.restitution_ball_wall": 0.5}.items():
        set_path(p, k, v)
    return p


def large_res100(p, viscosity):
    for k, v in {"mill.diameter_m": 0.221, "media.ball_diameter_m": 0.002, "simulation.resolution": 100,
                 "slurry.viscosity_pa_s": viscosity}.items():
        set_path(p, k, v)
    return p


def lower_drum_discs(n, drum_radius, ball_radius, seed, top=0.35):
    """n non-overlapping disc centres drawn uniformly (rejection sampling) in the drum below
    y = top * R, one radius clear of the wall; float32, shape (n, 2)."""
    rng = np.random.default_rng(seed)
    rmax = drum_radius - 1.05 * ball_radius
    pts = np.zeros((0, 2))
    min2 = (2.02 * ball_radius) ** 2
    while len(pts) < n:
        x, y = rng.uniform(-rmax, rmax), rng.uniform(-rmax, top * rmax)
        if x * x + y * y > rmax * rmax:
            continue
        if len(pts) and (((pts - (x, y)) ** 2).sum(axis=1) < min2).any():
            continue
        pts = np.vstack([pts, (x, y)])
    return pts.astype(np.float32)


# name -> (builder(backend) -> (params, initial balls or None), advance: list of ("frame"|"sub", count))
def cases():
    def realtime(b):
        return b.preset(b.params_default(), "realtime"), None

    def realtime_300(b):
        p = b.preset(b.params_default(), "realtime")
        set_path(p, "media.density_kg_m3", 7800.0)
        return p, lower_drum_discs(300, 0.0315, 0.001, seed=2024)

    return {
        "realtime_1_substep": (realtime, [("sub", 1)]),
        "realtime_10_frames": (realtime, [("frame", 10)]),
        "realtime_300_discs_5_frames": (realtime_300, [("frame", 5)]),
        "dem_500_10_frames": (lambda b: (dem_500(b.params_default()), None), [("frame", 10)]),
        "large_res100_mu1e-3_1_substep": (lambda b: (large_res100(b.params_default(), 1e-3), None), [("sub", 1)]),
        "large_res100_mu1e-1_1_substep": (lambda b: (large_res100(b.params_default(), 1e-1), None), [("sub", 1)]),
    }


def run_case(backend, name):
    """Runs one case; returns the record the fixture stores."""
    from milldynamics3_b200.sim import Simulation
    build, plan = cases()[name]
    p, balls = build(backend)
    s = Simulation(backend, p, initial_balls=balls)
    for kind, count in plan:
        for _ in range(count):
            if kind == "frame":
                s.step(1.0 / 60.0)
            else:
                s.step_fixed()
    nb, nf = s.counts()
    sc = s.scalars()
    rec = {"n_balls": int(nb), "n_fluid": int(nf), "state_hash": "%016x" % s.state_hash(True),
           "power_draw_w": float(sc.power_draw_w), "torque_nm": float(sc.torque_nm),
           "sim_time": float(sc.sim_time)}
    s.close()
    return rec
