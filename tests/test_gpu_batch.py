"""Batches (mg_batch_*): mills of different sizes and sub-step counts advanced in one launch per
frame give, mill by mill, exactly the results of the same mills stepped alone, and the oracle's."""
from __future__ import annotations

import numpy as np
import pytest

from milldynamics3_b200.batch import Batch, mix_params
from milldynamics3_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def _scalar_tuple(s):
    return (s.drum_angle, s.power_draw_w, s.torque_nm, s.collision_rate_per_s, s.dissipated_power_w,
            s.max_substep_displacement_over_diameter, s.coupling_clamp_hits, s.viscosity_iterations,
            s.mean_shear_rate_per_s, s.sim_time)


def _budget_tuple(e):
    return tuple(getattr(e, f) for f, _ in type(e)._fields_)


def _small_mix(backend, n, seed):
    ps, _ = mix_params(backend, 4 * n, seed=seed)
    d = [backend.derived(p) for p in ps]
    # the smallest mills of the draw (quick to check against the oracle), still of mixed sizes
    order = sorted(range(len(ps)), key=lambda i: d[i].eff_ball_count * d[i].effective_fluid_resolution ** 2)
    return [ps[i] for i in order[:n]]


def test_batch_matches_mills_stepped_alone(device):
    ps = _small_mix(device, 6, seed=3)
    subs = {device.derived(p).effective_substeps for p in ps}
    batch = Batch(device, ps)
    assert len(batch) == len(ps)
    batch.step_frames(2)
    sc = batch.scalars()
    for i, p in enumerate(ps):
        alone = Simulation(device, p)
        alone.step(1.0 / 60.0)
        alone.step(1.0 / 60.0)
        m = batch.mill(i)
        assert m.state_hash(True) == alone.state_hash(True), f"mill {i}"
        assert _scalar_tuple(sc[i]) == _scalar_tuple(alone.scalars()), f"mill {i} scalars"
        assert _budget_tuple(m.energy_budget()) == _budget_tuple(alone.energy_budget()), f"mill {i} budget"
        assert np.array_equal(m.stress_histogram_rate(), alone.stress_histogram_rate()), f"mill {i} stress"
        alone.close()
    assert len(subs) >= 1
    batch.close()


def test_batch_mill_matches_oracle(device, oracle):
    ps = _small_mix(device, 3, seed=5)
    batch = Batch(device, ps)
    batch.step_frames(1)
    for i, p in enumerate(ps):
        so = Simulation(oracle, p)
        so.step(1.0 / 60.0)
        assert batch.mill(i).state_hash(True) == so.state_hash(True), f"mill {i}"
    batch.close()


def test_batch_with_different_substep_counts_and_a_dry_mill(device):
    ps = _small_mix(device, 4, seed=7)
    dry = ps[0].copy()
    dry.slurry.enabled = 0
    ps = ps + [dry]
    batch = Batch(device, ps)
    batch.step_frames(1)
    alone = Simulation(device, dry)
    alone.step(1.0 / 60.0)
    assert batch.mill(len(ps) - 1).state_hash(True) == alone.state_hash(True)
    ms, n = batch.last_kernel_ms()
    assert ms > 0.0 and n == 1
    batch.close()


def test_block_size_does_not_change_results(device):
    """Every stage is an exact replay of the reference's order, so the block's thread count
    (128 to 1024) changes no result bit."""
    ps = _small_mix(device, 3, seed=19)
    hashes = []
    for bt in (512, 1024, 256, 128):
        batch = Batch(device, ps)
        batch.set_options(block_threads=bt)
        batch.step_frames(2)
        hashes.append([batch.mill(i).state_hash(True) for i in range(len(ps))])
        batch.close()
    assert hashes[0] == hashes[1] == hashes[2] == hashes[3]
