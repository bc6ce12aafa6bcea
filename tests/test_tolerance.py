"""The tolerance_probe gate (tolerance_probe.rs:11-27, 202-219, 330-446) as milldynamics3_b200.tolerance
restates it: gate rules, statistics, CSV layout, and a short run on the oracle."""
from __future__ import annotations

import math

import numpy as np
import pytest

from milldynamics3_b200 import tolerance as tp


def test_rel_gate_uses_two_sigma_or_two_percent():
    assert tp.judge(tp.REL, (100.0, 0.0), (101.9, 0.0)) == (pytest.approx(1.9), True)
    assert tp.judge(tp.REL, (100.0, 0.0), (102.1, 0.0))[1] is False
    # 2 sqrt(se_a^2 + se_b^2) = 2 * 5 = 10 beats the 2 % floor
    assert tp.judge(tp.REL, (100.0, 3.0), (109.0, 4.0))[1] is True
    assert tp.judge(tp.REL, (100.0, 3.0), (111.0, 4.0))[1] is False


def test_angle_gate_wraps_and_has_a_two_degree_floor():
    d, ok = tp.judge(tp.ANGLE, (359.0, 0.0), (1.0, 0.0))
    assert d == pytest.approx(2.0) and ok is True
    d, ok = tp.judge(tp.ANGLE, (1.0, 0.0), (358.5, 0.0))
    assert d == pytest.approx(-2.5) and ok is False


def test_energy_fraction_and_compression_gates():
    assert tp.judge(tp.ENERGY_FRACTION, (0.17, 0.0), (-0.19, 0.0))[1] is True    # 0.19 <= 0.187 + 0.005
    assert tp.judge(tp.ENERGY_FRACTION, (0.17, 0.0), (0.20, 0.0))[1] is False
    assert tp.judge(tp.COMPRESSION, (0.01, 0.0), (0.0111, 0.0))[1] is True       # <= 0.011 + 1e-4
    assert tp.judge(tp.COMPRESSION, (0.01, 0.0), (0.0112, 0.0))[1] is False


def test_nan_handling_and_informational_metrics():
    assert tp.judge(tp.REL, (math.nan, 0.0), (math.nan, 0.0)) == (0.0, True)
    d, ok = tp.judge(tp.REL, (1.0, 0.0), (math.nan, 0.0))
    assert math.isnan(d) and ok is False
    assert tp.judge(tp.INFO, (1.0, 0.0), (5.0, 0.0)) == (4.0, None)
    assert tp.judge(tp.INFO, (math.nan, 0.0), (5.0, 0.0))[1] is None


def test_mean_se_and_circular_mean():
    m, se = tp.mean_se([1.0, 2.0, 3.0, math.nan, math.inf])
    assert m == 2.0 and se == pytest.approx(math.sqrt(1.0 / 3.0))
    assert tp.mean_se([4.0]) == (4.0, 0.0)
    assert all(math.isnan(v) for v in tp.mean_se([math.nan]))
    assert tp.circular_mean_deg([350.0, 10.0]) == pytest.approx(0.0, abs=1e-9) or \
        tp.circular_mean_deg([350.0, 10.0]) == pytest.approx(360.0)
    assert tp.circular_mean_deg([80.0, 100.0]) == pytest.approx(90.0)
    assert math.isnan(tp.circular_mean_deg([]))
    assert math.isnan(tp.mean_or_nan([]))


def test_to_vertical_degrees_matches_metrics_rs_examples():
    # metrics.rs:262-274: atan2 ~220 deg maps to ~230 deg from vertical, ~18 deg to ~72, CCW
    assert tp.to_vertical_degrees(math.radians(220.0), 1.0) == pytest.approx(230.0, abs=1e-3)
    assert tp.to_vertical_degrees(math.radians(18.0), 1.0) == pytest.approx(72.0, abs=1e-3)
    assert tp.to_vertical_degrees(math.radians(18.0), -1.0) == pytest.approx(288.0, abs=1e-3)


def test_rust_exp_formatting_round_trips():
    cases = {1234.5: "1.2345e3", 0.001: "1e-3", 1.0: "1e0", -2.5e-7: "-2.5e-7", 0.0: "0e0",
             123456789.0: "1.23456789e8"}
    for x, want in cases.items():
        assert tp.rust_exp(x) == want
        assert float(want) == x
    assert tp.rust_exp(math.nan) == "NaN" and tp.rust_exp(math.inf) == "inf"
    x = 0.1 + 0.2
    assert float(tp.rust_exp(x)) == x


def test_csv_round_trip_and_compare(tmp_path):
    table = {("ship_fast", name): (1.0 + k, 0.01 * k) for k, (name, _) in enumerate(tp.METRICS)}
    table[("ship_fast", "toe_angle_deg")] = (math.nan, math.nan)
    path = tmp_path / "base.csv"
    tp.write_csv(str(path), table)
    lines = path.read_text().splitlines()
    assert lines[0] == "config,metric,mean,se" and lines[1].startswith("ship_fast,power_w,1e0,")
    back = tp.read_csv(str(path))
    assert back.keys() == table.keys()
    for k in table:
        a, b = table[k], back[k]
        assert (math.isnan(a[0]) and math.isnan(b[0])) or a == b
    out = []
    assert tp.compare(back, table, out.append) == 0
    worse = dict(table)
    worse[("ship_fast", "power_w")] = (1.5, 0.0)
    worse[("ship_fast", "compression_mean")] = (100.0, 0.0)
    out = []
    assert tp.compare(back, worse, out.append) == 2
    assert sum("FAIL" in l for l in out) == 2


def test_window_frames_follow_the_mill_speed(oracle):
    for cfg in tp.CONFIGS[:3]:
        p = tp.params_for(oracle, cfg, 1)
        rpm = oracle.derived(p).rpm
        s, m = tp.window_frames(oracle, p, 2.0, 3.0)
        assert abs(s - 2.0 * 60.0 / rpm * 60.0) <= 0.5 + 1e-3
        assert abs(m - 3.0 * 60.0 / rpm * 60.0) <= 0.5 + 1e-3


def test_short_probe_on_the_oracle(oracle):
    table = tp.run_all(oracle, seeds=2, settle_revs=0.02, measure_revs=0.05, only=["ship_fast"], batched=False)
    names = [n for n, _ in tp.METRICS]
    assert sorted(k[1] for k in table) == sorted(names)
    for n in ("power_w", "torque_nm", "impacts_per_ball_per_s", "compression_mean", "mean_shear_rate_per_s"):
        assert math.isfinite(table[("ship_fast", n)][0]), n
    assert table[("ship_fast", "power_w")][0] > 0.0
