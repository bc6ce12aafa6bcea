"""metrics::compute on the oracle (metrics.rs:195-711): the reference's own metrics tests
(metrics.rs:716-1200), restated over the C ABI, plus the consistency of the fields."""
from __future__ import annotations

import math

import numpy as np
import pytest

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Simulation


def to_vertical_degrees(atan2_rad, omega):
    # metrics.rs:275-279
    sign = -1.0 if omega >= 0.0 else 1.0
    return math.degrees(sign * (atan2_rad - math.pi / 2)) % 360.0


@pytest.mark.slow
def test_cascading_charge_toe_shoulder_in_the_acceptance_ranges(oracle):
    # metrics.rs:716-780: 1 m drum at 70 % of critical, 20 mm balls, 25 % fill, no lifters,
    # 300 balls (coarse-grained), 8 s of dry tumbling
    p = oracle.params_default()
    p.mill.diameter_m = 1.0
    p.mill.speed_mode = capi.SPEED_PERCENT_CRITICAL
    p.mill.speed_value = 70.0
    p.media.ball_diameter_m = 0.02
    p.media.fill_fraction = 0.25
    p.lifters.count = 0
    p.slurry.enabled = 0
    p.simulation.max_balls = 300
    p.simulation.coarse_graining_mode = 0  # Auto
    oracle.validate(p)
    s = Simulation(oracle, p)
    for _ in range(8 * 60):
        s.step(1.0 / 60.0)
    met = s.metrics()
    assert met.valid & capi.METRIC_TOE_SHOULDER
    omega = oracle.derived(p).omega
    toe = to_vertical_degrees(met.toe_angle_rad, omega)
    shoulder = to_vertical_degrees(met.shoulder_angle_rad, omega)
    assert 170.0 <= toe <= 270.0, toe
    assert 10.0 <= shoulder <= 100.0, shoulder


def test_realtime_mill_metrics_are_finite_and_consistent(oracle):
    # metrics.rs:966-1019 (debug checks finite and reasonable) and 1137-1159 (mean <= max)
    p = oracle.preset(oracle.params_default(), "realtime")
    s = Simulation(oracle, p)
    for _ in range(20):
        s.step(1.0 / 60.0)
    met = s.metrics()
    d = met.to_dict()
    for k, v in d.items():
        if isinstance(v, float):
            assert math.isfinite(v), k
    assert met.valid & capi.METRIC_CENTROID and met.valid & capi.METRIC_DENSITY
    assert met.mean_fluid_density_error_fraction <= met.max_fluid_density_error_fraction
    assert met.mean_fluid_compression_error_fraction <= met.max_fluid_compression_error_fraction
    assert 0.0 <= met.max_ball_overlap_fraction < 2.0 and 0.0 <= met.max_ball_wall_overlap_fraction < 2.0
    assert met.total_kinetic_energy_j > 0.0
    assert met.fluid_particle_count == s.counts()[1]
    assert met.drum_omega_rad_s == pytest.approx(oracle.derived(p).omega)
    # the centroid is the plain mean of the ball positions, below the drum centre
    x = s.balls()["x"]
    assert met.charge_centroid_m[1] < 0.0
    assert met.charge_centroid_m[0] == pytest.approx(float(np.mean(x[:, 0])), abs=1e-6)
    # the mixing index is mg_mixing_index's
    mi = s.mixing_index()
    assert (mi is None) == (not met.valid & capi.METRIC_MIXING)
    if mi is not None:
        assert met.mixing_index == mi
    # the pool sits at the bottom and has a plausible depth
    assert met.valid & capi.METRIC_POOL_DEPTH
    R = oracle.derived(p).radius_m
    assert 0.0 < met.pool_depth_m < 2.0 * R


def test_empty_populations_compute_gracefully_to_none(oracle):
    # metrics.rs:1093-1135: no balls and no fluid leave every Option field out
    p = oracle.params_default()
    p.slurry.enabled = 0
    s = Simulation(oracle, p, initial_balls=np.zeros((0, 2), np.float32))
    met = s.metrics()
    assert s.counts() == (0, 0)
    assert met.valid == 0
    assert met.total_kinetic_energy_j == 0.0
    assert met.max_ball_overlap_fraction == 0.0 and met.max_ball_wall_overlap_fraction == 0.0
    assert met.fluid_particle_count == 0
