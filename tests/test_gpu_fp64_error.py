"""The device's f32 path against the FP64 oracle: each output's error after one sub-step from a
common state (with the viscosity solve's inner products in f32 as the reference sums them, and in
f64), and the multi-second statistics gate: time-averaged power draw, torque, mixing index and
impact-energy histogram rate over 8 seeds within 2 % of the FP64 oracle's."""
from __future__ import annotations

import json
import multiprocessing as mp
import os

import pytest

import fp64_report as FR

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("preset", ["realtime", "accuracy"])
def test_per_output_error_against_the_fp64_oracle(device, oracle, oracle64, preset):
    p = device.preset(device.params_default(), preset)
    errs = FR.single_step_errors([device, oracle], oracle64, p, warm_frames=10, cg_fp64=(0, 1))
    print("\nFP64 error table (%s): %s" % (preset, json.dumps(errs, sort_keys=True)))
    # the device is the parity oracle bit for bit, so its error is the f32 restatement's own
    assert errs["0/cg_fp64=0"] == errs["1/cg_fp64=0"]
    for mode in ("0/cg_fp64=0", "0/cg_fp64=1"):
        e = errs[mode]
        assert e["ball_x"]["rel"] < 1e-5 and e["fluid_x"]["rel"] < 1e-5, (mode, e)
        assert e["ball_v"]["rel"] < 1e-4 and e["fluid_v"]["rel"] < 1e-4, (mode, e)


def test_eight_seed_statistics_within_two_percent_of_the_fp64_oracle(device):
    p = device.preset(device.params_default(), "realtime")
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(8, os.cpu_count() or 1)) as pool:
        gate, f32, f64 = FR.ensemble_gate(device, None, p, list(range(1, 9)), settle_s=1.0, measure_s=3.0,
                                          pool=pool)
    print("\nFP64 gate (realtime, seeds 1-8, 1 s settle, 3 s window): %s" % json.dumps(gate))
    for k, (a, r, rel) in gate.items():
        assert rel < 0.02, (k, a, r, rel)
