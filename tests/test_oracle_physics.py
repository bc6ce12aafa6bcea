"""Oracle pins against the reference's physics unit tests (pbf.rs, dem.rs, coupling.rs, lib.rs),
run through the oracle's C API with the same setups and assertions."""
from __future__ import annotations

import pytest

import scenarios as S


def test_fluid_stays_inside_the_drum_and_finite(oracle):
    S.fluid_stays_inside_the_drum_and_finite(oracle)


def test_dye_is_conserved(oracle):
    S.dye_is_conserved(oracle)


def test_extreme_velocity_is_bounded(oracle):
    S.extreme_velocity_is_bounded(oracle)


def test_non_finite_fluid_particle_is_reset(oracle):
    S.non_finite_fluid_particle_is_reset(oracle)


def test_non_finite_ball_does_not_contaminate_fluid(oracle):
    S.non_finite_ball_does_not_contaminate_fluid(oracle)


def test_head_on_collision_conserves_momentum(oracle):
    S.head_on_collision_conserves_momentum(oracle)


def test_restitution_bounce(oracle):
    S.restitution_bounce(oracle)


def test_step_fixed_matches_step(oracle):
    S.step_fixed_matches_step(oracle)


def test_drum_angle_kinematics(oracle):
    S.drum_angle_kinematics(oracle)


def test_momentum_exchange_is_symmetric(oracle):
    S.momentum_exchange_is_symmetric(oracle)


def test_seeding_counts(oracle):
    S.seeding_counts(oracle)


def test_realtime_frame_is_deterministic_and_finite(oracle):
    """The `perf_probe` determinism property (examples/perf_probe.rs:230-262): identical runs
    give identical FNV-1a state hashes."""
    from helpers import params
    from milldynamics3_b200.sim import Simulation
    import numpy as np

    hashes = []
    for _ in range(2):
        s = Simulation(oracle, params(oracle, preset="realtime"))
        s.step(1.0 / 60.0)
        hashes.append(s.state_hash(True))
        assert np.all(np.isfinite(s.balls()["x"])) and np.all(np.isfinite(s.fluid()["x"]))
    assert hashes[0] == hashes[1]
