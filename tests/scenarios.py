"""Backend-generic restatements of the reference's physics unit tests (same setups, same
assertions). Each scenario takes a Backend (the oracle or the device library) so the identical
check runs on both: tests/test_oracle_physics.py pins the oracle with them, and
tests/test_gpu_physics.py runs them through the CUDA library."""
from __future__ import annotations

import math

import numpy as np

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Simulation

from helpers import ball_inertia, ball_mass, dem_state, params, still_drum

F = np.float32


def fluid_only_sim(b, radius_m=0.5, fill=0.15, res=20, **kw):
    """FluidParticles::seed_lattice(&slurry, radius_m, res, &[], 0.0) via a ball-free Simulation
    (the media diameter only keeps effective_fluid_resolution at `res`)."""
    p = params(b, **{"mill.diameter_m": 2 * radius_m, "media.fill_fraction": 0.0,
                     "media.ball_diameter_m": 2 * radius_m / res, "slurry.fill_fraction": fill,
                     "simulation.resolution": res, **kw})
    return Simulation(b, p), p


# pbf.rs:3087 fluid_stays_inside_the_drum_and_finite
def fluid_stays_inside_the_drum_and_finite(b, steps=480):
    s, p = fluid_only_sim(b)
    drum = still_drum(0.5)
    for _ in range(steps):
        s.fluid_step_coupled(drum, 0.0, p.slurry, 3, 1.0 / 240.0)
    x = s.fluid()["x"]
    assert np.all(np.isfinite(x))
    assert np.all(np.linalg.norm(x, axis=1) <= 0.5 * 1.05)
    return s


# pbf.rs:3111 dye_is_conserved_per_particle_pure_advection
def dye_is_conserved(b):
    s, p = fluid_only_sim(b)
    before = s.fluid()["dye"].copy()
    for _ in range(60):
        s.fluid_step_coupled(still_drum(0.5), 0.0, p.slurry, 3, 1.0 / 240.0)
    assert np.array_equal(s.fluid()["dye"], before)
    assert (before == 0).any() and (before == 1).any()


# pbf.rs:3360 an_injected_extreme_velocity_is_bounded_within_one_sub_step
def extreme_velocity_is_bounded(b):
    s, p = fluid_only_sim(b)
    f = s.fluid()
    v = f["v"].copy()
    v[0] = (1.0e6, 0.0)
    s.set_fluid(f["x"], v, f["dye"])
    s.fluid_step_coupled(still_drum(0.5), 0.0, p.slurry, 3, 1.0 / 240.0)
    v_max = 5.0 * (0.0 + math.sqrt(4.0 * 9.81 * 0.5))
    vv = s.fluid()["v"]
    assert np.all(np.isfinite(vv))
    assert np.all(np.linalg.norm(vv, axis=1) <= v_max * 1.001)


def _one_ball_sim(b, count, radius_m=0.5):
    """DemState::new(&EffectiveMedia{d=0.05, rho=7800, count}, radius_m, 1) plus an empty fluid of
    resolution 20 (h = 2 * radius_m / 20)."""
    r = 0.025
    j = count * r * r / (0.82 * radius_m * radius_m)
    p = params(b, **{"mill.diameter_m": 2 * radius_m, "mill.speed_value": 0.0, "media.ball_diameter_m": 0.05,
                     "media.density_kg_m3": 7800.0, "media.fill_fraction": j, "slurry.fill_fraction": 0.0,
                     "simulation.resolution": 20})
    s = Simulation(b, p)
    assert s.counts()[0] == count
    return s, p


# pbf.rs:3384 a_non_finite_fluid_particle_is_reset_and_never_reaches_the_ball_coupling
def non_finite_fluid_particle_is_reset(b):
    s, p = _one_ball_sim(b, 1)
    s.set_balls([(0.35, 0.0)])
    fm = s.fluid_material()
    assert s.counts()[1] == 0
    s.set_fluid([(math.nan, 0.0)], [(0.0, 0.0)], [0.0])
    s.set_fluid_material(fm.particle_mass, fm.h, fm.rest_density)
    slurry = p.slurry.copy()
    slurry.fill_fraction = 0.0
    imp, _ = s.fluid_step_coupled(still_drum(0.5), 0.0, slurry, 3, 1.0 / 240.0)
    f = s.fluid()
    assert np.all(np.isfinite(f["x"][0])) and np.all(np.isfinite(f["v"][0]))
    assert np.linalg.norm(f["x"][0]) <= 0.5 * 1.05
    assert np.linalg.norm(imp.impulses[0]) < 1e-6


# pbf.rs:3433 a_non_finite_ball_position_does_not_contaminate_the_fluid
def non_finite_ball_does_not_contaminate_fluid(b):
    s, p = _one_ball_sim(b, 4)
    fs, _ = fluid_only_sim(b)
    f = fs.fluid()
    fm = fs.fluid_material()
    s.set_fluid(f["x"], f["v"], f["dye"])
    s.set_fluid_material(fm.particle_mass, fm.h, fm.rest_density)
    bl = s.balls()
    x = bl["x"].copy()
    x[0] = (math.inf, math.inf)
    s.set_balls(x, bl["v"], bl["theta"], bl["omega"])
    slurry = p.slurry.copy()
    slurry.fill_fraction = 0.15
    s.fluid_step_coupled(still_drum(0.5), 0.0, slurry, 3, 1.0 / 240.0)
    f2 = s.fluid()
    assert np.all(np.isfinite(f2["x"])) and np.all(np.isfinite(f2["v"]))


# dem.rs:1289 two_balls_head_on_collision_conserves_momentum
def head_on_collision_conserves_momentum(b):
    r = 0.05
    m = ball_mass(2 * r, 7800.0)
    s = dem_state(b, [(-0.5, 0.0), (0.5, 0.0)], [(2.0, 0.0), (-2.0, 0.0)], r, m)
    media = b.params_default().media
    media.restitution_ball_ball = 0.9
    media.friction_ball_ball = 0.0
    media.friction_ball_ball_static = 0.0
    media.rolling_friction = 0.0
    drum = still_drum(1000.0)
    v = s.balls()["v"]
    px0 = F(m) * (v[0, 0] + v[1, 0])
    for _ in range(600):
        s.dem_step(drum, 0.0, media, 4, 1.0 / 480.0)
    bl = s.balls()
    px1 = F(m) * (bl["v"][0, 0] + bl["v"][1, 0])
    assert abs(px1 - px0) / max(abs(px0), 1e-9) < 0.05
    assert bl["x"][1, 0] > bl["x"][0, 0] + 2 * r * 0.9


# dem.rs:1236 ball_bounces_with_restitution_e_squared_height_ratio
def restitution_bounce(b):
    rd, r, e, h0 = 10.0, 0.05, 0.8, 0.5
    m = ball_mass(2 * r, 7800.0)
    start_y = -(F(rd) - F(r)) + F(h0)
    s = dem_state(b, [(0.0, start_y)], [(0.0, 0.0)], r, m)
    media = b.params_default().media
    media.restitution_ball_wall = e
    media.friction_ball_wall = 0.0
    media.friction_ball_wall_static = 0.0
    media.rolling_friction = 0.0
    drum = still_drum(rd)
    max_h, bounced, settled = -np.inf, False, 0
    for _ in range(20000):
        s.dem_step(drum, 0.0, media, 4, 1.0 / 480.0)
        bl = s.balls()
        height = (F(rd) - np.linalg.norm(bl["x"][0])) - F(r)
        if not bounced:
            if bl["v"][0, 1] > 0 and height < h0 * 0.5:
                bounced = True
        else:
            max_h = max(max_h, height)
            if bl["v"][0, 1] <= 0:
                settled += 1
                if settled > 5:
                    break
    assert bounced
    assert abs(max_h - e * e * h0) / (e * e * h0) < 0.25


# lib.rs:595 step_fixed_called_substeps_times_matches_one_step_call_at_1x
def step_fixed_matches_step(b):
    p = params(b, **{"media.fill_fraction": 0.0, "slurry.enabled": 0})
    n = b.derived(p).effective_substeps
    a = Simulation(b, p)
    a.step(1.0 / 60.0)
    c = Simulation(b, p)
    c.reset_frame_stats()
    for _ in range(n):
        c.step_fixed()
    sa, sc = a.scalars(), c.scalars()
    assert abs(sa.sim_time - sc.sim_time) < 1e-9 and abs(sa.drum_angle - sc.drum_angle) < 1e-6


# lib.rs drum-angle kinematics tests (step_advances_drum_angle_at_correct_rate, wraps, clockwise)
def drum_angle_kinematics(b):
    p = params(b, **{"mill.speed_value": 60.0, "media.fill_fraction": 0.0, "slurry.enabled": 0})
    s = Simulation(b, p)
    s.step(0.25)
    assert abs(s.scalars().drum_angle - math.pi / 2) < 1e-3
    s2 = Simulation(b, p)
    s2.step(1.5)
    assert 0.0 <= s2.scalars().drum_angle < 2 * math.pi
    p.mill.direction = capi.DIR_CW
    s3 = Simulation(b, p)
    s3.step(0.25)
    assert abs(s3.scalars().drum_angle - (2 * math.pi - math.pi / 2)) < 1e-3


# coupling.rs:672 ball_fluid_momentum_exchange_is_symmetric_when_unclamped
def momentum_exchange_is_symmetric(b, warm=60):
    radius_m = 1.0
    r = 0.025
    j = 6 * r * r / (0.82 * radius_m * radius_m)
    p = params(b, **{"mill.diameter_m": 2.0, "mill.speed_value": 0.0, "media.ball_diameter_m": 0.05,
                     "media.density_kg_m3": 4000.0, "media.fill_fraction": j, "slurry.fill_fraction": 0.3,
                     "simulation.resolution": 20, "simulation.seed": 3})
    s = Simulation(b, p)
    assert s.counts()[0] == 6
    drum = still_drum(radius_m)
    media = b.params_default().media
    for _ in range(warm):
        s.coupling_step_recorded(drum, 0.0, media, p.slurry, 4, 3, 1.0 / 240.0)
    imp, _ = s.fluid_step_coupled(drum, 0.0, p.slurry, 3, 1.0 / 240.0)
    if imp.clamp_hits == 0:
        total = imp.impulses.astype(np.float64).sum(0)
        expected = -imp.fluid_momentum_change.astype(np.float64)
        assert np.linalg.norm(total - expected) / max(np.linalg.norm(expected), 1e-9) < 1e-3
    return s


# lib.rs:696 new_seeds_the_expected_number_of_balls, and the realtime seeding
def seeding_counts(b):
    p = params(b)
    s = Simulation(b, p)
    assert s.counts()[0] == b.derived(p).eff_ball_count
    rt = Simulation(b, params(b, preset="realtime"))
    nb, nf = rt.counts()
    assert nb == 407 and 700 < nf < 900
