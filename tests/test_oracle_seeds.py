"""Seed sweeps on the oracle: the reference's batch.rs tests (batch.rs:196-262) and a check of the
sweep's frame logic against a loop over the public Simulation API."""
from __future__ import annotations

import math

import pytest

from milldynamics3_b200 import capi, seeds
from milldynamics3_b200.sim import MillError, Simulation


def dry(b):
    p = b.params_default()
    p.slurry.enabled = 0
    return p


def test_value_names(oracle):
    names = seeds.value_names(oracle)
    assert len(names) == capi.SEED_VALUES == len(set(names))
    assert names[0] == "specific_power_w_per_kg"
    assert names[16] == "window_specific_power_w_per_kg"
    assert names[-1] == "window_effective_power_per_ball_w.thr5"


def test_run_seed_is_deterministic_and_seeds_differ(oracle):
    # batch.rs:203-219
    p = dry(oracle)
    a = seeds.run_seed(oracle, p, 1, 1.0, 1.0)
    b = seeds.run_seed(oracle, p, 1, 1.0, 1.0)
    c = seeds.run_seed(oracle, p, 2, 1.0, 1.0)
    assert a.values == b.values
    assert a.values != c.values
    assert len(a.names) == len(a.values)
    assert a.get("specific_power_w_per_kg") > 0.0
    assert abs(a.window_s - 0.6) < 0.02
    assert a.coarse_graining_factor == 1.0


@pytest.mark.slow
def test_exact_window_power_agrees_with_the_smoothed_mean(oracle):
    # batch.rs:221-231
    r = seeds.run_seed(oracle, dry(oracle), 1, 2.0, 2.0)
    smoothed = r.get("specific_power_w_per_kg")
    exact = r.get("window_specific_power_w_per_kg")
    assert abs(smoothed - exact) / exact < 0.2, (smoothed, exact)


def test_combine_gives_mean_and_standard_error(oracle):
    # batch.rs:233-248, through the C entry point (every one of the 23 slots gets the same value)
    names = seeds.value_names(oracle)
    mk = lambda v: seeds.SeedResult(0, 1.0, 1.0, names, [v] * capi.SEED_VALUES, 0.0)
    c = seeds.combine(oracle, [mk(1.0), mk(2.0), mk(3.0)])
    assert c.seeds == 3
    assert all(abs(m - 2.0) < 1e-12 for m in c.mean)
    assert all(abs(s - 1.0 / math.sqrt(3.0)) < 1e-12 for s in c.std_err)
    one = seeds.combine(oracle, [mk(5.0)])
    assert one.mean[0] == 5.0 and one.std_err[0] == 0.0
    with pytest.raises(MillError):
        seeds.combine(oracle, [])


def test_drift_is_zero_for_flat_and_detects_a_ramp(oracle):
    # batch.rs:250-257
    assert seeds.drift_per_rev(oracle, [2.0] * 10, 10.0) == 0.0
    y = [1.0 + 0.1 * i for i in range(10)]
    assert abs(seeds.drift_per_rev(oracle, y, 10.0) - 1.0 / 1.45) < 1e-9
    assert seeds.drift_per_rev(oracle, [3.0], 10.0) == 0.0


def test_rejects_bad_arguments(oracle):
    p = dry(oracle)
    with pytest.raises(MillError):
        seeds.run_seed(oracle, p, 1, 1.0, 0.5)
    with pytest.raises(MillError):
        seeds.run_seed(oracle, p, 1, -1.0, 1.0)
    q = p.copy()
    q.mill.speed_value = 0.0
    with pytest.raises(MillError):
        seeds.run_seed(oracle, q, 1, 0.0, 1.0)


def test_sweep_matches_a_loop_over_the_public_api(oracle):
    """run_seed's frame logic (batch.rs:55-107) restated here over Simulation.step/stress_metrics."""
    p = dry(oracle)
    p.simulation.seed = 7
    warm_rev, meas_rev = 0.5, 1.0
    omega = float(oracle.derived(p).omega)
    rev_s = 2.0 * math.pi / abs(omega)
    warm = round(warm_rev * rev_s * 60.0)
    meas = max(round(meas_rev * rev_s * 60.0), 1)
    frame = 1.0 / 60.0
    s = Simulation(oracle, p)
    for _ in range(warm):
        s.step(frame)
    start = s.stress_metrics()
    acc = [0.0] * 16
    powers = []
    for _ in range(meas):
        s.step(frame)
        m = s.stress_metrics()
        v = [m.specific_power_w_per_kg, m.wall_power_per_ball_w, m.impacts_total_per_ball_per_s,
             m.mean_se_scaled_drop, m.mean_se_scaled_shear, m.stress_intensity_scaled,
             *list(m.impacts_per_ball_per_s), *list(m.effective_power_per_ball_w)]
        acc = [a + x for a, x in zip(acc, v)]
        powers.append(m.wall_power_per_ball_w)
    end = s.stress_metrics()
    r = seeds.run_seed(oracle, p, 7, warm_rev, meas_rev)
    assert r.window_s == pytest.approx(meas / 60.0, rel=1e-6)
    assert r.values[:16] == [a / meas for a in acc]
    w = r.window_s
    assert r.values[16] == (end.cumulative_specific_energy_j_per_kg - start.cumulative_specific_energy_j_per_kg) / w
    for q in range(6):
        d = end.cumulative_effective_energy_per_ball_j[q] - start.cumulative_effective_energy_per_ball_j[q]
        assert r.values[17 + q] == d / w
    assert r.power_drift_rel_per_rev == seeds.drift_per_rev(oracle, powers, rev_s * 60.0)
