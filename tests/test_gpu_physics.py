"""The reference's physics unit tests (pbf.rs, dem.rs, coupling.rs, lib.rs), restated against the
C ABI of the CUDA library with the same setups and assertions as the oracle pins, plus
bit-for-bit agreement with the oracle on the same scenario where it is deterministic."""
from __future__ import annotations

import numpy as np
import pytest

import scenarios as S

pytestmark = pytest.mark.gpu


def test_fluid_stays_inside_the_drum_and_finite(device, oracle):
    sd = S.fluid_stays_inside_the_drum_and_finite(device, steps=120)
    so = S.fluid_stays_inside_the_drum_and_finite(oracle, steps=120)
    assert sd.state_hash(True) == so.state_hash(True)


def test_dye_is_conserved(device):
    S.dye_is_conserved(device)


def test_extreme_velocity_is_bounded(device):
    S.extreme_velocity_is_bounded(device)


def test_non_finite_fluid_particle_is_reset(device):
    S.non_finite_fluid_particle_is_reset(device)


def test_non_finite_ball_does_not_contaminate_fluid(device):
    S.non_finite_ball_does_not_contaminate_fluid(device)


def test_head_on_collision_conserves_momentum(device):
    S.head_on_collision_conserves_momentum(device)


def test_restitution_bounce(device):
    S.restitution_bounce(device)


def test_step_fixed_matches_step(device):
    S.step_fixed_matches_step(device)


def test_drum_angle_kinematics(device):
    S.drum_angle_kinematics(device)


def test_momentum_exchange_is_symmetric(device, oracle):
    sd = S.momentum_exchange_is_symmetric(device, warm=30)
    so = S.momentum_exchange_is_symmetric(oracle, warm=30)
    assert sd.state_hash(True) == so.state_hash(True)


def test_seeding_counts(device):
    S.seeding_counts(device)
