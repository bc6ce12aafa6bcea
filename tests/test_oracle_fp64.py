"""The FP64 oracle (the oracle's restatement built with Real = double): it loads behind the same
C API, steps the realtime mill from the parity oracle's state, and the parity oracle's f32
outputs after one sub-step stay within f32-sized errors of it (the per-output error table the
device path inherits: the device equals the parity oracle bit for bit)."""
from __future__ import annotations

import fp64_report as FR


def test_fp64_oracle_steps_the_realtime_mill_from_the_f32_state(oracle, oracle64):
    p = oracle.preset(oracle.params_default(), "realtime")
    errs = FR.single_step_errors([oracle], oracle64, p, warm_frames=10)
    e = errs["0/cg_fp64=0"]
    # positions: the f32 rounding of one step's motion; velocities: the f32 noise of the
    # iterative solves (density loop, Gauss-Seidel sweeps, CG); both far below the 1e-5 budget
    # for positions, and velocities of the same order as it
    assert e["ball_x"]["rel"] < 1e-6 and e["fluid_x"]["rel"] < 1e-6, e
    assert e["ball_v"]["rel"] < 1e-4 and e["fluid_v"]["rel"] < 1e-4, e
    for k, v in e.items():
        assert v["rel"] < 1e-3, (k, v)


def test_fp64_oracle_differs_from_the_f32_oracle(oracle, oracle64):
    # the two builds are different arithmetic (not the same library twice)
    from milldynamics3_b200.sim import Simulation
    p = oracle.preset(oracle.params_default(), "realtime")
    a, b = Simulation(oracle, p), Simulation(oracle64, p)
    FR.copy_state(a, b)
    a.step_fixed()
    b.step_fixed()
    assert a.state_hash(True) != b.state_hash(True)
