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

from milldynamics3_b200 import workloads


def dem_500(p):
    """The DEM-only configuration with 500 discs (the 0.45 m drum)."""
    return workloads.dem_only_params(p, diameter_m=0.45)


def large_res100(p, viscosity):
    return workloads.large_params(p, 100, viscosity)


# name -> (builder(backend) -> (params, initial balls or None), advance: list of ("frame"|"sub", count))
def cases():
    def realtime(b):
        return b.preset(b.params_default(), "realtime"), None

    realtime_300 = workloads.realtime_300

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
