"""Backend-generic restatements of more of the reference's own unit tests for the sub-step path:
the drag, buoyancy, wall-work, cohesion, adhesion, hydrostatic and viscosity tests of pbf.rs, the
adhesion, clamp-rate and energy-invariant tests of coupling.rs, the rolling, lifter-work,
energy, density and tunnelling tests of dem.rs, the energy tests of lib.rs and the mixing-index
tests of metrics.rs. Each function takes a Backend (the oracle or the device library), builds the
reference test's state through the C ABI with the same numbers (f32 arithmetic where the
reference computes in f32), runs the same calls and makes the same assertions; the device tests
also compare the returned quantities with the oracle's bit for bit where the run is
deterministic. Each function's comment names the reference test (file:line)."""
from __future__ import annotations

import math

import numpy as np

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Simulation

from helpers import ball_inertia, ball_mass, lifters, params, still_drum

F = np.float32
GRAVITY = F(9.81)
TAU_F = F(2.0 * math.pi)


def _len(v):
    v = np.asarray(v, F)
    return np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1])


def empty_state(b, **kw):
    """A handle with no balls and no fluid (slurry on, zero fills), ready for a hand-built state
    (the reference tests build `Balls` and `FluidParticles` literals)."""
    p = params(b, **{"media.fill_fraction": 0.0, "slurry.fill_fraction": 0.0, **kw})
    s = Simulation(b, p)
    assert s.counts() == (0, 0)
    return s, p


def set_state(s, ball_x=None, r=None, m=None, inertia=None, true_r=None, ball_v=None, ball_omega=None,
              fluid_x=None, fluid_v=None, particle_mass=None, h=None, rho0=None):
    if ball_x is not None:
        bx = np.asarray(ball_x, F).reshape(-1, 2)
        s.set_balls(bx, None if ball_v is None else np.asarray(ball_v, F).reshape(-1, 2), None,
                    None if ball_omega is None else np.asarray(ball_omega, F))
        s.set_ball_material(r, m, inertia, true_r)
    if fluid_x is not None:
        fx = np.asarray(fluid_x, F).reshape(-1, 2)
        fv = np.zeros_like(fx) if fluid_v is None else np.asarray(fluid_v, F).reshape(-1, 2)
        s.set_fluid(fx, fv, np.zeros(len(fx), F))
        s.set_fluid_material(particle_mass, h, rho0)


def lattice_material(radius_m, resolution, rho0=1000.0):
    """FluidParticles::seed_lattice's h and particle mass (pbf.rs:1051-1068), in f32."""
    dx = F(radius_m) / F(max(resolution, 1))
    h = F(2.0) * dx
    row_h = dx * (np.sqrt(F(3.0)) * F(0.5))
    return float(F(rho0) * (dx * row_h)), float(h), float(rho0)


def slurry_of(b, **kw):
    s = b.params_default().slurry.copy()
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def media_of(b, **kw):
    m = b.params_default().media.copy()
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def drum(radius, omega=0.0, lift=None):
    return still_drum(radius, omega, lifters(0) if lift is None else lift)


# ---------------------------------------------------------------- pbf.rs: drag (step 6.5)

def ball_in_uniform_fluid_patch(b, ball_radius_m, ball_density, rho0, fluid_velocity, offset=(0.0, 0.0),
                                co_rotate_omega=None):
    """pbf.rs:2613-2676 ball_in_uniform_fluid_patch (+ the buoyancy tests' offset and co-rotation)."""
    r = F(ball_radius_m)
    mass = ball_mass(2.0 * ball_radius_m, ball_density)
    inertia = ball_inertia(mass, ball_radius_m)
    dx = r * F(4.0)
    h = F(2.0) * dx
    particle_mass = F(rho0) * dx * dx
    half_span = r + h
    exclude = F(1.01) * (r + F(0.25) * h)
    n = int(math.ceil(float(F(2.0) * half_span / dx)))
    xs = []
    for iy in range(-n, n + 1):
        for ix in range(-n, n + 1):
            p = np.array([F(ix) * dx, F(iy) * dx], F)
            dist = _len(p)
            if half_span >= dist >= exclude:
                xs.append(p)
    fx = np.array(xs, F)
    off = np.array(offset, F)
    fx = fx + off
    if co_rotate_omega is not None:
        w = F(co_rotate_omega)
        fv = np.stack([w * -fx[:, 1], w * fx[:, 0]], axis=1).astype(F)
    else:
        fv = np.tile(np.array(fluid_velocity, F), (len(fx), 1))
    s, _ = empty_state(b)
    set_state(s, ball_x=[off], r=float(r), m=mass, inertia=inertia, true_r=float(r),
              fluid_x=fx, fluid_v=fv, particle_mass=float(particle_mass), h=float(h), rho0=rho0)
    return s, mass


# pbf.rs:2677 ball_drag_matches_two_dimensional_stokes_scaling
def drag_matches_stokes_scaling(b):
    d = drum(2.0)
    fluid_velocity, dt = 0.3, 1.0 / 240.0
    out = {}
    for mu in (10.0, 100.0):
        slurry = slurry_of(b, viscosity_pa_s=mu, fill_fraction=0.0, wettability=0.0)
        s, _ = ball_in_uniform_fluid_patch(b, 0.03, 6000.0, slurry.density_kg_m3, (fluid_velocity, 0.0))
        imp, _ = s.fluid_step_coupled(d, 0.0, slurry, 1, dt)
        out[mu] = float(_len(imp.impulses[0]))
        s.close()
    for mu, impulse in out.items():
        expected = float(F(4.0) * F(math.pi) * F(mu) * F(fluid_velocity) * F(dt))
        assert abs(impulse - expected) / expected < 0.5, (mu, impulse, expected)
    assert out[100.0] > out[10.0] * 3.0
    return out


# pbf.rs:2743 ball_drag_gains_form_drag_at_high_relative_speed_and_low_viscosity
def drag_gains_form_drag(b):
    d = drum(2.0)
    mu, v, dt = 0.001, 2.0, 1.0 / 240.0
    slurry = slurry_of(b, viscosity_pa_s=mu, fill_fraction=0.0, wettability=0.0)
    s, mass = ball_in_uniform_fluid_patch(b, 0.01, 6000.0, slurry.density_kg_m3, (v, 0.0))
    imp, _ = s.fluid_step_coupled(d, 0.0, slurry, 1, dt)
    impulse = float(_len(imp.impulses[0]))
    pure_stokes = float(F(4.0) * F(math.pi) * F(mu) * F(v) * F(dt))
    assert impulse > pure_stokes * 100.0
    assert impulse <= float(F(mass) * F(v)) * 1.0001
    s.close()
    return impulse


# pbf.rs:2785 ball_drag_never_overshoots_the_local_fluid_velocity
def drag_never_overshoots(b):
    d = drum(2.0)
    dt = 1.0 / 240.0
    slurry = slurry_of(b, viscosity_pa_s=200.0, fill_fraction=0.0, wettability=0.0)
    s, mass = ball_in_uniform_fluid_patch(b, 0.005, 6000.0, slurry.density_kg_m3, (1.0, 0.0))
    imp, _ = s.fluid_step_coupled(d, 0.0, slurry, 1, dt)
    assert imp.clamp_hits == 0
    new_vx = F(0.0) + imp.impulses[0, 0] / F(mass)
    assert 0.0 <= new_vx <= 1.0 * 1.001
    s.close()
    return float(new_vx)


# ---------------------------------------------------------------- pbf.rs: buoyancy (step 6.6)

def _buoyancy_slurry(b):
    return slurry_of(b, viscosity_pa_s=0.0, ball_no_slip=0.0, wettability=0.0, surface_tension_n_m=0.0,
                     wall_no_slip=0.0, fill_fraction=0.0)


# pbf.rs:2819 buoyancy_is_purely_vertical_at_rest_and_inward_while_the_fluid_itself_co_rotates
def buoyancy_vertical_at_rest_inward_when_co_rotating(b):
    slurry = _buoyancy_slurry(b)
    dt = 1.0 / 480.0

    def impulse_x(omega, co_rotate):
        s, _ = ball_in_uniform_fluid_patch(b, 0.01, 6000.0, slurry.density_kg_m3, (0.0, 0.0), offset=(0.3, 0.0),
                                           co_rotate_omega=omega if co_rotate else None)
        imp, _ = s.fluid_step_coupled(drum(10.0, omega), 0.0, slurry, 1, dt)
        s.close()
        return float(imp.impulses[0, 0])

    still = impulse_x(0.0, False)
    spinning = impulse_x(4.0, True)
    assert abs(still) < 1e-6, still
    assert spinning < -1e-6, spinning
    return still, spinning


# pbf.rs:2886 buoyancy_ignores_drum_rotation_when_the_pool_itself_is_still
def buoyancy_ignores_drum_rotation_for_a_still_pool(b):
    slurry = _buoyancy_slurry(b)
    s, _ = ball_in_uniform_fluid_patch(b, 0.01, 6000.0, slurry.density_kg_m3, (0.0, 0.0), offset=(0.3, 0.0))
    imp, _ = s.fluid_step_coupled(drum(10.0, 4.0), 0.0, slurry, 1, 1.0 / 480.0)
    s.close()
    assert abs(float(imp.impulses[0, 0])) < 1e-4
    return float(imp.impulses[0, 0])


# ---------------------------------------------------------------- pbf.rs: wall, coupling reach, hydrostatics

def fluid_only(b, radius_m, resolution, **slurry_kw):
    """FluidParticles::seed_lattice(&slurry, radius_m, resolution, &[], 0.0) through a ball-free
    handle (the ball diameter only keeps effective_fluid_resolution at `resolution`)."""
    kw = {"mill.diameter_m": 2 * radius_m, "media.fill_fraction": 0.0,
          "media.ball_diameter_m": 2 * radius_m / resolution, "simulation.resolution": resolution}
    kw.update({"slurry." + k: v for k, v in slurry_kw.items()})
    p = params(b, **kw)
    s = Simulation(b, p)
    assert s.counts()[0] == 0
    return s, p.slurry.copy()


# pbf.rs:2938 wall_drag_does_positive_work_while_spinning_and_none_at_rest
def wall_drag_work(b):
    kw = dict(viscosity_pa_s=5.0, wall_no_slip=1.0, wettability=0.0, surface_tension_n_m=0.0, fill_fraction=0.2)
    out = []
    for omega in (0.0, 3.0):
        s, slurry = fluid_only(b, 0.3, 24, **kw)
        total = F(0.0)
        for _ in range(60):
            _, st = s.fluid_step_coupled(drum(0.3, omega), 0.0, slurry, 3, 1.0 / 240.0)
            total = F(total + F(st.wall_work_j))
        out.append(float(total))
        s.close()
    assert out[0] == 0.0, out
    assert out[1] > 0.0, out
    return out


# pbf.rs:2985 coupling_finds_ball_neighbours_beyond_two_radii
def coupling_finds_neighbours_beyond_two_radii(b):
    r = F(0.01)
    slurry = slurry_of(b, viscosity_pa_s=50.0, fill_fraction=0.0)
    dx = r * F(1.5)
    h = F(2.0) * dx
    assert r + F(0.5) * h > F(2.0) * r
    mass = ball_mass(2.0 * float(r), 6000.0)
    s, _ = empty_state(b)
    set_state(s, ball_x=[(0.0, 0.0)], r=float(r), m=mass, inertia=ball_inertia(mass, float(r)), true_r=float(r),
              fluid_x=[(r + F(0.5) * h, 0.0)], fluid_v=[(1.0, 0.0)],
              particle_mass=float(F(slurry.density_kg_m3) * dx * dx), h=float(h), rho0=slurry.density_kg_m3)
    imp, _ = s.fluid_step_coupled(drum(2.0), 0.0, slurry, 1, 1.0 / 240.0)
    s.close()
    assert float(_len(imp.impulses[0])) > 1e-9
    return imp.impulses[0].copy()


# pbf.rs:3032 hydrostatic_column_settles_near_rest_density
def hydrostatic_column(b, steps=240):
    s, slurry = fluid_only(b, 0.5, 20, fill_fraction=0.25)
    assert s.counts()[1] > 20
    for _ in range(steps):
        s.fluid_step_coupled(drum(0.5), 0.0, slurry, 3, 1.0 / 240.0)
    dens = s.fluid_densities()
    x = s.fluid()["x"]
    h = F(s.fluid_material().h)
    max_y = x[:, 1].max()
    margin = F(1.5) * h
    checked = 0
    for i in range(len(x)):
        if min(F(0.5) - _len(x[i]), max_y - x[i, 1]) < margin:
            continue
        checked += 1
        assert abs(dens[i] - slurry.density_kg_m3) / slurry.density_kg_m3 < 0.1, (i, dens[i])
    assert checked > 5
    return s


# ---------------------------------------------------------------- pbf.rs: the viscosity solve

# pbf.rs:3133 viscosity_solve_is_a_no_op_at_zero_viscosity
def viscosity_noop_at_zero(b):
    s, slurry = fluid_only(b, 0.5, 20, fill_fraction=0.2, viscosity_pa_s=0.0)
    _, st = s.fluid_step_coupled(drum(0.5), 0.0, slurry, 3, 1.0 / 240.0)
    assert st.viscosity_iterations == 0
    s.close()


# pbf.rs:3175 viscosity_solve_stays_finite_and_converges_at_high_viscosity_and_rotation
def viscosity_converges_at_high_viscosity_and_rotation(b, steps=480):
    s, slurry = fluid_only(b, 0.5, 20, fill_fraction=0.2, viscosity_pa_s=200.0)
    omega, dt = F(6.0), F(1.0 / 240.0)
    d = drum(0.5, float(omega))
    angle = F(0.0)
    iters = []
    for k in range(steps):
        _, st = s.fluid_step_coupled(d, float(angle), slurry, 3, float(dt))
        angle = F(np.fmod(angle + omega * dt, TAU_F))  # rem_euclid of a non-negative angle
        assert st.viscosity_iterations < 50, (k, st.viscosity_iterations)
        assert math.isfinite(st.mean_shear_rate_per_s) and st.mean_shear_rate_per_s >= 0.0, k
        assert np.all(np.isfinite(s.fluid()["v"])), k
        iters.append(st.viscosity_iterations)
    return s, iters


def _checkerboard_baseline(b):
    """pbf.rs:3229-3268: a puddle settled once at 0.5 Pa s, then a column-parity x-velocity
    perturbation of +-2 m/s."""
    radius_m, res = 0.5, 20
    dx = F(radius_m) / F(res)
    s, slurry = fluid_only(b, radius_m, res, fill_fraction=0.2, viscosity_pa_s=0.5)
    for _ in range(240):
        s.fluid_step_coupled(drum(radius_m), 0.0, slurry, 3, 1.0 / 240.0)
    f = s.fluid()
    x, v = f["x"].copy(), f["v"].copy()
    col = np.round(x[:, 0] / dx).astype(np.int64)  # f32::round: halves away from zero
    col = np.where(np.abs(x[:, 0] / dx - np.trunc(x[:, 0] / dx)) == 0.5,
                   (np.trunc(x[:, 0] / dx) + np.sign(x[:, 0])).astype(np.int64), col)
    v[:, 0] = v[:, 0] + np.where(col % 2 == 0, F(2.0), F(-2.0)).astype(F)
    mat = s.fluid_material()
    s.close()
    return x, v, f["dye"].copy(), (mat.particle_mass, mat.h, mat.rest_density), slurry


def _perturbation_energy(v):
    e = np.add.accumulate((v[:, 0] * v[:, 0]).astype(F), dtype=F)[-1]
    return F(e / F(len(v)))


def _decay_run(b, base, mu, steps=20):
    x, v, dye, mat, slurry = base
    s, _ = fluid_only(b, 0.5, 20, fill_fraction=0.2)
    s.set_fluid(x, v, dye)  # viscous_guess starts empty (Vec::new())
    s.set_fluid_material(*mat)
    sl = slurry.copy()
    sl.viscosity_pa_s = mu
    for _ in range(steps):
        s.fluid_step_coupled(drum(0.5), 0.0, sl, 3, 1.0 / 240.0)
    e = _perturbation_energy(s.fluid()["v"])
    s.close()
    return e


# pbf.rs:3149 viscosity_keeps_mattering_between_100_and_200_pa_s (checkerboard_shear_decay_rate)
def viscosity_matters_between_100_and_200(b):
    base = _checkerboard_baseline(b)
    e0 = _perturbation_energy(base[1])
    rates = []
    for mu in (100.0, 200.0):
        e1 = _decay_run(b, base, mu)
        ratio = min(max(float(F(e1 / max(e0, F(1e-12)))), 1e-6), 1.0)
        rates.append(-0.5 * math.log(ratio) / (20 * (1.0 / 240.0)))
    assert rates[1] > rates[0] * 1.05, rates
    return rates


# pbf.rs:3269-3355 higher_viscosity_damps_a_high_frequency_perturbation_more_across_the_whole_range
def higher_viscosity_damps_more(b):
    base = _checkerboard_baseline(b)
    res = [float(_decay_run(b, base, mu)) for mu in (0.5, 2.0, 10.0, 50.0, 100.0, 200.0)]
    for a, c in zip(res, res[1:]):
        assert c < a, res
    return res


# ---------------------------------------------------------------- pbf.rs: cohesion (step 3.6a)

# pbf.rs:3463 cohesion_pulls_two_isolated_fluid_particles_together_only_when_surface_tension_is_positive
def cohesion_two_particles(b):
    out = []
    for sigma in (0.0, 0.072):
        s, slurry = fluid_only(b, 0.5, 20, fill_fraction=0.0, wall_no_slip=0.0, viscosity_pa_s=0.0,
                               surface_tension_n_m=sigma)
        assert s.counts()[1] == 0
        pm, h, rho0 = lattice_material(0.5, 20, slurry.density_kg_m3)
        sep = F(0.6) * F(h)
        set_state(s, fluid_x=[(F(-0.5) * sep, 0.0), (F(0.5) * sep, 0.0)], particle_mass=pm, h=h, rho0=rho0)
        s.fluid_step_coupled(drum(0.5), 0.0, slurry, 1, 1.0 / 240.0)
        out.append((s.fluid()["v"].copy(), F(s.fluid_material().particle_mass)))
        s.close()
    (v_off, _), (v_on, mass) = out
    assert v_off[0, 0] == 0.0 and v_off[1, 0] == 0.0
    assert v_on[0, 0] > 1e-6 and v_on[1, 0] < -1e-6
    assert abs(mass * (v_on[0, 0] + v_on[1, 0])) < 1e-6
    return v_off, v_on


# ---------------------------------------------------------------- coupling.rs: adhesion

def _one_fluid_one_ball(b, ball_radius_m, radius_m, resolution, fluid_x, wettability):
    slurry = slurry_of(b, fill_fraction=0.0, wall_no_slip=0.0, viscosity_pa_s=0.0, surface_tension_n_m=0.0,
                       wettability=wettability)
    s, _ = empty_state(b)
    pm, h, rho0 = lattice_material(radius_m, resolution, slurry.density_kg_m3)
    mass = ball_mass(2.0 * ball_radius_m, 7800.0)
    set_state(s, ball_x=[(0.0, 0.0)], r=ball_radius_m, m=mass, inertia=ball_inertia(mass, ball_radius_m),
              true_r=ball_radius_m, fluid_x=[fluid_x], particle_mass=pm, h=h, rho0=rho0)
    imp, _ = s.fluid_step_coupled(drum(radius_m), 0.0, slurry, 1, 1.0 / 240.0)
    v = s.fluid()["v"][0].copy()
    s.close()
    return v, imp.impulses[0].copy(), F(pm)


# coupling.rs:347-433 adhesion_pulls_a_ball_and_nearby_fluid_together_only_when_wettability_is_positive
def adhesion_only_when_wettable(b):
    fx = (F(0.1) + F(0.0075), 0.0)
    v_off, imp_off, _ = _one_fluid_one_ball(b, 0.1, 1.0, 200, fx, 0.0)
    assert v_off[0] == 0.0
    assert imp_off[0] == 0.0 and imp_off[1] == 0.0
    v_on, imp_on, mass = _one_fluid_one_ball(b, 0.1, 1.0, 200, fx, 1.0)
    assert v_on[0] < -1e-6 and imp_on[0] > 1e-9
    assert abs(mass * v_on[0] + imp_on[0]) < 1e-6
    return v_on, imp_on


# coupling.rs:436-500 adhesion_range_is_capped_at_twice_the_ball_radius_regardless_of_fluid_resolution
def adhesion_range_is_capped(b):
    _, imp, _ = _one_fluid_one_ball(b, 0.01, 1.0, 10, (F(3.0) * F(0.01) + F(0.001), 0.0), 1.0)
    assert abs(imp[0]) < 1e-6, imp
    return imp


# ---------------------------------------------------------------- coupling.rs: clamp rate, energy

def charge_sim(b, count, ball_d, radius_m, density=None, resolution=20, slurry_fill=0.15, seed=1, **kw):
    """DemState::new(&EffectiveMedia{d, rho, count}, radius_m, seed) plus FluidParticles::seed_lattice
    around its balls at `resolution`, through Simulation::new (same seeding)."""
    r = ball_d / 2
    j = count * r * r / (0.82 * radius_m * radius_m)
    p = params(b, **{"mill.diameter_m": 2 * radius_m, "media.ball_diameter_m": ball_d, "media.fill_fraction": j,
                     "slurry.fill_fraction": slurry_fill, "simulation.resolution": resolution,
                     "simulation.seed": seed, **({"media.density_kg_m3": density} if density else {}), **kw})
    s = Simulation(b, p)
    assert s.counts()[0] == count, s.counts()
    return s, p


# coupling.rs:720-786 cascading_charge_clamp_rate (the 50 and 200 Pa s tests, :788 and :806)
def cascading_clamp_rate(b, viscosity, settle=3 * 240, measure=2 * 240):
    radius_m, omega, dt = 0.5, F(3.0), F(1.0 / 240.0)
    d = drum(radius_m, float(omega))
    media = media_of(b, ball_diameter_m=0.02, fill_fraction=0.25)
    s, p = charge_sim(b, 150, 0.02, radius_m, resolution=20, **{"slurry.viscosity_pa_s": viscosity})
    slurry = slurry_of(b, fill_fraction=0.15, viscosity_pa_s=viscosity)
    angle = F(0.0)
    for _ in range(settle):
        s.coupling_step_recorded(d, float(angle), media, slurry, 4, 3, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
    hits = 0
    for _ in range(measure):
        imp, _ = s.fluid_step_coupled(d, float(angle), slurry, 3, float(dt))
        hits += imp.clamp_hits
        s.dem_step(d, float(angle), media, 4, float(dt), external=imp, cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
    rate = hits / (150.0 * measure)
    assert rate < 0.10, rate
    return s, rate


def ball_energy(s, bl=None):
    """dem.rs:253-261 mechanical_energy_j in f32, summed in ball order."""
    bl = s.balls() if bl is None else bl
    mat = s.ball_material()
    m, inertia = F(mat.mass), F(mat.inertia)
    v, om, x = bl["v"], bl["omega"], bl["x"]
    t = np.empty((len(v), 3), F)
    t[:, 0] = F(0.5) * m * (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1])
    t[:, 1] = F(0.5) * inertia * om * om
    t[:, 2] = m * GRAVITY * x[:, 1]
    return F(np.add.accumulate(t.reshape(-1), dtype=F)[-1]) if len(v) else F(0.0)


def fluid_energy(s, fl=None):
    """pbf.rs:1005-1013 mechanical_energy_j in f32, summed in particle order."""
    fl = s.fluid() if fl is None else fl
    m = F(s.fluid_material().particle_mass)
    v, x = fl["v"], fl["x"]
    t = np.empty((len(v), 2), F)
    t[:, 0] = F(0.5) * m * (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1])
    t[:, 1] = m * GRAVITY * x[:, 1]
    return F(np.add.accumulate(t.reshape(-1), dtype=F)[-1]) if len(v) else F(0.0)


def full_system_energy_invariant(b, p, settle_s, measure_s):
    """coupling.rs:1000-1123 settle_and_measure_full_system_energy_invariant: worst per-sub-step
    margin of wall work + tolerance - dE (balls + fluid), max ball speed, max centroid distance
    over the RMS spread."""
    s = Simulation(b, p)
    d = b.derived(p)
    radius_m = F(p.mill.diameter_m) * F(0.5)
    omega = F(d.omega)
    dr = capi.Drum()
    dr.radius_m, dr.omega, dr.lifters = float(radius_m), float(omega), p.lifters
    sub_dt = F(F(1.0) / (F(60.0) * F(d.effective_substeps)))
    angle = F(0.0)
    cap = 4 * s.counts()[0] + 256
    for _ in range(int(F(settle_s) / sub_dt)):
        s.coupling_step_recorded(dr, float(angle), p.media, p.slurry, p.simulation.dem_iterations,
                                 p.simulation.pbf_iterations, float(sub_dt), cap=cap)
        angle = F(np.fmod(angle + omega * sub_dt, TAU_F))
    mass = F(s.ball_material().mass)
    tol = max(float(F(1e-2) * mass * max(F(omega * radius_m) ** 2, F(1.0))), 15.0)
    worst = math.inf
    e_prev = F(ball_energy(s) + fluid_energy(s))
    vmax, dmax, sumsq, nsamp = 0.0, 0.0, 0.0, 0
    for _ in range(int(F(measure_s) / sub_dt)):
        fs, ds, _ = s.coupling_step_recorded(dr, float(angle), p.media, p.slurry, p.simulation.dem_iterations,
                                             p.simulation.pbf_iterations, float(sub_dt), cap=cap)
        angle = F(np.fmod(angle + omega * sub_dt, TAU_F))
        bl = s.balls()
        e_now = F(ball_energy(s, bl) + fluid_energy(s))
        worst = min(worst, float(F(ds.wall_work_j) + F(fs.wall_work_j)) + tol - float(e_now - e_prev))
        e_prev = e_now
        vmax = max(vmax, float(_len(bl["v"]).max()))
        c = bl["x"].astype(np.float64).mean(0)
        dist = np.sqrt(((bl["x"] - c) ** 2).sum(1))
        sumsq += float((dist * dist).sum())
        nsamp += len(dist)
        dmax = max(dmax, float(dist.max()))
    rms = math.sqrt(sumsq / max(nsamp, 1))
    s.close()
    return worst, vmax, (dmax / rms if rms > 1e-6 else 0.0)


def _realtime_150_auto(b, **kw):
    return params(b, **{"simulation.max_balls": 150, "simulation.coarse_graining_mode": capi.CG_AUTO,
                        "simulation.resolution": 15, **kw})


# coupling.rs:930 low_fill_cataracting_charge_does_not_gain_energy_from_the_fluid
def low_fill_cataracting_energy(b, settle_s=5.0, measure_s=8.0):
    p = _realtime_150_auto(b, **{"mill.diameter_m": 1.0, "mill.speed_mode": capi.SPEED_RPM, "mill.speed_value": 30.0,
                                 "mill.direction": capi.DIR_CCW, "media.fill_fraction": 0.10})
    b.validate(p)
    worst, vmax, ratio = full_system_energy_invariant(b, p, settle_s, measure_s)
    assert worst >= 0.0, worst
    assert vmax < 15.0, vmax
    assert ratio < 10.0, ratio
    return worst, vmax, ratio


# coupling.rs:1149 coupled_charge_never_gains_more_energy_than_the_wall_supplies
def coupled_charge_energy(b, settle_s=3.0, measure_s=8.0):
    p = _realtime_150_auto(b)
    b.validate(p)
    worst, _, _ = full_system_energy_invariant(b, p, settle_s, measure_s)
    assert worst >= 0.0, worst
    return worst


# ---------------------------------------------------------------- dem.rs

def dem_only(b, max_balls, seed=None, lift=None, **kw):
    """DemState::new(&params.effective_media(), radius, params.simulation.seed) through a dry
    Simulation::new (same seeding)."""
    p = params(b, **{"slurry.enabled": 0, "simulation.max_balls": max_balls,
                     "simulation.coarse_graining_mode": capi.CG_AUTO, **kw})
    if seed is not None:
        p.simulation.seed = seed
    if lift is not None:
        p.lifters = lift
    b.validate(p)
    return Simulation(b, p), p


def _drum_of(b, p):
    d = b.derived(p)
    dr = capi.Drum()
    dr.radius_m = float(F(p.mill.diameter_m) * F(0.5))
    dr.omega = float(d.omega)
    dr.lifters = p.lifters
    return dr


# dem.rs:1334 ball_resting_on_rotating_wall_settles_into_rolling_without_slip
def rolling_without_slip(b):
    from helpers import dem_state
    rd, omega, r = 10.0, 0.5, 0.05
    m = ball_mass(2 * r, 7800.0)
    s = dem_state(b, [(0.0, -(F(rd) - F(r)))], [(0.0, 0.0)], r, m)
    d = drum(rd, omega)
    media = b.params_default().media
    for _ in range(5 * 480):
        s.dem_step(d, 0.0, media, 4, 1.0 / 480.0)
    bl = s.balls()
    x, v, w = bl["x"][0], bl["v"][0], F(bl["omega"][0])
    # drum.sdf_world(x, 0) for a smooth circle: the SDF R - |p| grows inward, so n_hat = -p / |p|
    # (up to the central-difference noise the reference itself notes); wall velocity omega * perp(p)
    n_hat = -x / _len(x)
    t_hat = np.array([-n_hat[1], n_hat[0]], F)
    pc = x - F(r) * n_hat
    v_wall = F(omega) * np.array([-pc[1], pc[0]], F)
    slip = float(np.dot(v - v_wall, t_hat) - F(r) * w)
    wall_speed = float(_len(v_wall))
    assert abs(slip) < 0.05 * max(wall_speed, 1e-6), (slip, wall_speed, w)
    return s


# dem.rs:1382 lifter_normal_force_contributes_to_wall_work
def lifter_wall_work(b):
    r, rd, omega = 0.02, 0.5, F(6.0)
    lift = lifters(6, 0.03, 0.05, 0.03, 0.0)
    d = drum(rd, float(omega), lift)
    media = b.params_default().media
    media.rolling_friction = 0.0
    j = 40 * r * r / (0.82 * rd * rd)
    p = params(b, **{"slurry.enabled": 0, "mill.diameter_m": 2 * rd, "media.ball_diameter_m": 2 * r,
                     "media.density_kg_m3": 6000.0, "media.fill_fraction": j, "simulation.seed": 42})
    s = Simulation(b, p)
    assert s.counts()[0] == 40
    dt = F(1.0 / 960.0)
    angle, total, any_work = F(0.0), F(0.0), False
    for _ in range(2 * 960):
        st, _ = s.dem_step(d, float(angle), media, 4, float(dt), cap=1024)
        total = F(total + F(st.wall_work_j))
        angle = F(np.fmod(angle + omega * dt, TAU_F))
        any_work = any_work or abs(st.wall_work_j) > 1e-9
    assert any_work
    assert total > 0.0, total
    return float(total)


# dem.rs:1784 total_energy_never_increases_in_a_still_drum
def energy_never_increases_in_still_drum(b):
    s, p = dem_only(b, 300, **{"mill.diameter_m": 1.0, "mill.speed_mode": capi.SPEED_RPM, "mill.speed_value": 0.0,
                                "media.fill_fraction": 0.30, "lifters.count": 0})
    d = drum(0.5)
    for _ in range(240):
        s.dem_step(d, 0.0, p.media, p.simulation.dem_iterations, 1.0 / 240.0, cap=4096)
    mat = s.ball_material()
    nb = s.counts()[0]
    tol = float(F(1e-4) * F(mat.mass) * F(nb) * F(9.81) * F(0.5))
    e_prev = ball_energy(s)
    worst = -math.inf
    for _ in range(4 * 240):
        s.dem_step(d, 0.0, p.media, p.simulation.dem_iterations, 1.0 / 240.0, cap=4096)
        e_now = ball_energy(s)
        worst = max(worst, float(e_now - e_prev))
        e_prev = e_now
    assert worst <= tol, (worst, tol)
    return worst


def _max_pair_overlap(s):
    from milldynamics3_b200.sim import probe_candidate_pairs
    r = F(s.ball_material().radius)
    x = s.balls()["x"]
    rc, pairs = None, None
    cell = max(float(F(2.0) * r * F(1.05)), 1e-6)
    pr = probe_candidate_pairs(s.b.lib, x, cell)
    rc, pairs = pr[0], pr[1]
    assert rc == 0
    worst = F(0.0)
    for i, j in pairs.reshape(-1, 2):
        dist = _len(x[i] - x[j])
        worst = max(worst, F(max(F(2.0) * r - dist, F(0.0)) / r))
    return float(worst)


def _cascading_1m(b, max_balls, lift_count=0):
    return dem_only(b, max_balls, **{"mill.diameter_m": 1.0, "mill.speed_mode": capi.SPEED_RPM,
                                      "mill.speed_value": 30.0, "mill.direction": capi.DIR_CCW,
                                      "media.fill_fraction": 0.30, "lifters.count": lift_count})


# dem.rs:1968 a_cascading_charge_stays_dense
def cascading_charge_stays_dense(b):
    s, p = _cascading_1m(b, 400)
    d = _drum_of(b, p)
    omega, dt = F(d.omega), F(1.0 / 240.0)
    angle = F(0.0)
    radius = F(d.radius_m)
    for step in range(10 * 240):
        s.dem_step(d, float(angle), p.media, p.simulation.dem_iterations, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
        if step % 240 != 239 or step < 3 * 240:
            continue
        assert _max_pair_overlap(s) < 0.7, step
        assert float(_len(s.balls()["x"]).min()) > 0.05 * float(radius), step
    return s


def cascading_density_samples(b):
    """dem.rs:1968's run: (largest ball-ball overlap, closest ball to the centre) once a second
    from t = 4 s to 10 s."""
    s, p = _cascading_1m(b, 400)
    d = _drum_of(b, p)
    omega, dt = F(d.omega), F(1.0 / 240.0)
    angle = F(0.0)
    over, mind = [], []
    for step in range(10 * 240):
        s.dem_step(d, float(angle), p.media, p.simulation.dem_iterations, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
        if step % 240 == 239 and step >= 3 * 240:
            over.append(_max_pair_overlap(s))
            mind.append(float(_len(s.balls()["x"]).min()))
    s.close()
    return over, mind


# dem.rs:2060 a_cataracting_charge_with_lifters_never_tunnels_through_a_lifter
def lifters_never_tunnel(b, sdf_lib, seconds=20):
    """sdf_lib: the oracle library, whose restated Drum::sdf_world (geometry.rs:79-114) measures the
    ball-wall overlap the reference test computes with max_ball_wall_overlap_fraction."""
    s, p = _cascading_1m(b, 400, lift_count=8)
    d = _drum_of(b, p)
    omega, dt = F(d.omega), F(1.0 / 240.0)
    angle = F(0.0)
    worst = 0.0
    r = F(s.ball_material().radius)
    for step in range(seconds * 240):
        s.dem_step(d, float(angle), p.media, p.simulation.dem_iterations, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
        if step < 5 * 240:
            continue
        sdf = wall_sdf(sdf_lib, d, s.balls()["x"], angle)
        overlap = float((np.maximum(r - sdf, F(0.0)) / r).max())
        worst = max(worst, overlap)
        assert overlap < 1.0, (step, overlap)
    return worst


def wall_sdf(lib, d, x, angle):
    """Drum::sdf_world distances of the points x (the oracle's restatement)."""
    import ctypes
    out = np.empty(len(x), F)
    dd, nx, ny = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    for k in range(len(x)):
        lib.sdf_world(ctypes.byref(d), float(x[k, 0]), float(x[k, 1]), float(angle), ctypes.byref(dd),
                      ctypes.byref(nx), ctypes.byref(ny))
        out[k] = dd.value
    return out


# dem.rs:2130 dissipated_energy_is_never_materially_negative_while_cascading
def dissipation_never_negative(b):
    s, p = _cascading_1m(b, 400)
    d = _drum_of(b, p)
    omega, dt = F(d.omega), F(1.0 / 240.0)
    angle = F(0.0)
    for _ in range(3 * 240):
        s.dem_step(d, float(angle), p.media, p.simulation.dem_iterations, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
    mass = F(s.ball_material().mass)
    tol = float(F(1e-3) * mass * max(F(omega * F(d.radius_m)) ** 2, F(1.0)))
    worst = math.inf
    for _ in range(5 * 240):
        st, _ = s.dem_step(d, float(angle), p.media, p.simulation.dem_iterations, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
        worst = min(worst, st.dissipated_energy_j)
        assert st.dissipated_energy_j >= -tol, (st.dissipated_energy_j, tol)
    assert math.isfinite(worst)
    return worst


# ---------------------------------------------------------------- lib.rs

# lib.rs:761 steady_cascading_charge_never_gains_more_energy_than_the_wall_supplies
def steady_cascading_energy(b):
    s, p = dem_only(b, 150, **{"mill.diameter_m": 1.0, "mill.speed_mode": capi.SPEED_PERCENT_CRITICAL,
                                "mill.speed_value": 70.0, "mill.direction": capi.DIR_CCW,
                                "media.ball_diameter_m": 0.02, "media.fill_fraction": 0.25, "lifters.count": 0})
    d = _drum_of(b, p)
    omega, dt = F(d.omega), F(1.0 / 240.0)
    angle = F(0.0)
    for _ in range(3 * 240):
        s.dem_step(d, float(angle), p.media, p.simulation.dem_iterations, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
    mass = F(s.ball_material().mass)
    tol = float(F(1e-3) * mass * max(F(omega * F(d.radius_m)) ** 2, F(1.0)))
    e_prev = ball_energy(s)
    worst = -math.inf
    for _ in range(5 * 240):
        st, _ = s.dem_step(d, float(angle), p.media, p.simulation.dem_iterations, float(dt), cap=4096)
        angle = F(np.fmod(angle + omega * dt, TAU_F))
        e_now = ball_energy(s)
        delta = float(e_now - e_prev)
        assert delta <= float(st.wall_work_j) + tol, (delta, st.wall_work_j, tol)
        worst = max(worst, delta - float(st.wall_work_j))
        e_prev = e_now
    return worst


# lib.rs:1205 energy_budget_is_finite_and_the_two_torque_readings_agree
def energy_budget_torque_readings(b):
    p = params(b, **{"simulation.resolution": 15, "simulation.max_balls": 100,
                     "simulation.coarse_graining_mode": capi.CG_AUTO})
    b.validate(p)
    omega = float(b.derived(p).omega)
    s = Simulation(b, p)
    for _ in range(30):
        s.step(1.0 / 60.0)
    s.reset_energy_budget()
    for _ in range(60):
        s.step(1.0 / 60.0)
    e = s.energy_budget()
    for k in ("shaft_work_j", "ball_contact_dissipation_j", "fluid_wall_slip_j", "fluid_viscous_j",
              "fluid_clamp_removed_j", "interface_created_j", "delta_mechanical_j", "unattributed_j"):
        assert math.isfinite(getattr(e, k)), k
    assert abs(e.elapsed_s - 1.0) < 1e-3
    from_impulse = omega * e.fluid_wall_angular_impulse
    assert abs(e.fluid_wall_work_j - from_impulse) <= 0.01 * abs(e.fluid_wall_work_j) + 1e-9
    return s, e


# ---------------------------------------------------------------- metrics.rs

# metrics.rs:888 mixing_index_starts_low_and_increases_under_tumbling
def mixing_index_increases(b, frames=4 * 60):
    p = params(b, **{"slurry.dye_pattern": capi.DYE_LEFT_RIGHT, "simulation.max_balls": 150,
                     "simulation.coarse_graining_mode": capi.CG_AUTO, "simulation.resolution": 20})
    s = Simulation(b, p)
    initial = s.mixing_index()
    assert initial is not None and 0.0 <= initial <= 1.0 and initial < 0.2, initial
    for _ in range(frames):
        s.step(1.0 / 60.0)
    later = s.mixing_index()
    assert later is not None and 0.0 <= later <= 1.0 and later > initial, (initial, later)
    return s, initial, later


# metrics.rs:921 mixing_index_weights_by_cell_particle_count_not_cell_count
def mixing_index_weights_by_count(b):
    s, _ = empty_state(b, **{"mill.diameter_m": 2.0, "mill.speed_value": 0.0})
    x = np.zeros((102, 2), F)
    dye = np.full(102, 0.5, F)
    x[100] = (-0.99, -0.99)
    dye[100] = 0.0
    x[101] = (0.99, 0.99)
    dye[101] = 1.0
    s.set_fluid(x, np.zeros_like(x), dye)
    s.set_fluid_material(1.0, 0.01, 1000.0)
    m = s.mixing_index()
    s.close()
    assert m is not None and m > 0.9, m
    return m


# ---------------------------------------------------------------- branches the tests above miss

# dem.rs:674-706 (step 2.5, wall CCD): a ball whose predicted end-of-step position lies deeper in
# the wall than one bounded recovery pass can absorb is held at its time of impact plus a skin.
def wall_ccd_clamps_a_fast_ball(b):
    from helpers import dem_state
    rd, r = 10.0, 0.05
    m = ball_mass(2 * r, 7800.0)
    # 12 m/s toward the floor from 1 cm above it: the predicted step (5 cm at dt = 1/240) ends
    # 0.8 r beyond the wall, past the 0.8 r (2 r * MAX_RECOVERY_FRACTION) the projection absorbs
    s = dem_state(b, [(0.0, -(F(rd) - F(r) - F(0.01)))], [(0.0, -12.0)], r, m)
    media = b.params_default().media
    st, recs = s.dem_step(drum(rd), 0.0, media, 4, 1.0 / 240.0, cap=64)
    ctr = s.last_step_stats()[2]
    assert ctr.ccd_clamps == 1, ctr.to_dict()
    x = s.balls()["x"][0]
    assert float(_len(x)) < rd  # the centre never crossed the wall
    return s, st, [bytes(r_) for r_ in recs]


# pbf.rs:2146-2153 with slurry.rheology = Bingham: the shear rates (pbf.rs:800-849) and the
# regularised effective viscosity (pbf.rs:851-868) feed the Morris weights. A yield stress adds
# viscosity (mu_eff >= mu), so a checkerboard perturbation decays faster than in the Newtonian
# fluid of the same plastic viscosity.
def bingham_damps_more_than_newtonian(b):
    base = _checkerboard_baseline(b)
    x, v, dye, mat, slurry = base
    out = []
    for rheology, tau in ((capi.RHEOLOGY_NEWTONIAN, 0.0), (capi.RHEOLOGY_BINGHAM, 20.0)):
        sl = slurry.copy()
        sl.rheology, sl.yield_stress_pa = rheology, tau
        out.append(float(_decay_run(b, (x, v, dye, mat, sl), 2.0)))
    assert out[1] < out[0], out
    return out


def bingham_realtime_mill(b, frames=2):
    """The realtime mill with a Bingham slurry (20 Pa yield stress), a few frames."""
    p = params(b, preset="realtime", **{"slurry.rheology": capi.RHEOLOGY_BINGHAM, "slurry.yield_stress_pa": 20.0})
    s = Simulation(b, p)
    for _ in range(frames):
        s.step(1.0 / 60.0)
    fs = s.last_step_stats()[0]
    assert np.all(np.isfinite(s.fluid()["v"])) and fs.viscosity_iterations > 0
    return s
