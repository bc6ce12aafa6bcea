"""Backend-generic restatements of surface.rs's unit tests (surface.rs:437-777: same setups, same
assertions) over Simulation::fluid_surface / build_field, plus the states the device parity tests
compare bit for bit. Each scenario takes a Backend (the oracle or the device library)."""
from __future__ import annotations

import math

import numpy as np

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Simulation, unflatten_polygons

from helpers import params, still_drum
from scenarios import fluid_only_sim

F = np.float32
G = capi.SURFACE_GRID


def shoelace_area(poly):
    """surface.rs:750-759 (f32 accumulation in point order)"""
    s = F(0.0)
    n = len(poly)
    for i in range(n):
        a, b = poly[i], poly[(i + 1) % n]
        s = F(s + F(F(a[0] * b[1]) - F(b[0] * a[1])))
    return float(abs(F(s * F(0.5))))


def surface_sim(b, fill=0.2, res=24, lifter_count=0, radius_m=0.5):
    """FluidParticles::seed_lattice(&slurry, 0.5, 24, &[], 0.0) in a drum with `lifter_count`
    default-shaped lifters (surface.rs:522-537 and 719-733)."""
    s, p = fluid_only_sim(b, radius_m=radius_m, fill=fill, res=res, **{"lifters.count": lifter_count})
    drum = still_drum(radius_m, lifters=p.lifters)
    return s, p, drum


def settle(s, p, drum, steps=120):
    for _ in range(steps):
        s.fluid_step_coupled(drum, 0.0, p.slurry, 3, 1.0 / 240.0)


def spin_up(s, p, omega=6.0):
    """surface.rs:586-602: a smooth drum at omega rad/s for 1 s of 1/240 s steps. The handle's own
    drum angle stays 0; a smooth drum's SDF does not depend on the angle."""
    drum = still_drum(0.5, omega=omega)
    dt = F(1.0 / 240.0)
    angle = F(0.0)
    for _ in range(int(1.0 / dt)):
        s.fluid_step_coupled(drum, float(angle), p.slurry, 3, float(dt))
        angle = F(np.fmod(F(angle + F(F(omega) * dt)), F(2 * math.pi)))


def points_inside(polys, radius_m=0.5):
    for poly in polys:
        r = np.hypot(poly[:, 0].astype(np.float64), poly[:, 1].astype(np.float64))
        assert np.all(r <= radius_m + 1e-4), f"contour point outside the drum: {poly[np.argmax(r)]}"


# surface.rs:438-443 splat_kernel_is_zero_outside_radius_and_positive_inside, through build_field:
# one particle on a grid point adds splat_kernel(0) = 1 there, positive values inside the splat
# radius and nothing at grid points at or beyond it.
def splat_kernel_zero_outside_radius(b):
    s, p, _ = surface_sim(b, fill=0.0, res=24)
    m = s.fluid_material()
    cell = F(F(2.0 * 0.5) / F(G - 1))
    gi = gj = 70
    x = F(F(-0.5) + F(F(gi) * cell))
    y = F(F(-0.5) + F(F(gj) * cell))
    s.set_fluid(np.array([[x, y]], F))
    field, _ = s.surface_field()
    assert field[gj, gi] == 1.0
    radius = F(1.5) * F(m.h)
    ii, jj = np.meshgrid(np.arange(G), np.arange(G))
    gx = F(-0.5) + ii.astype(F) * cell
    gy = F(-0.5) + jj.astype(F) * cell
    r2 = (gx - x) ** 2 + (gy - y) ** 2
    assert np.all(field[r2 >= radius * radius * 1.0001] == 0.0)
    assert np.all(field[r2 < radius * radius * 0.9999] > 0.0)


# surface.rs:446-502 build_field_interior_value_matches_analytic_phi_full
def interior_value_matches_phi_full(b):
    radius_m, resolution = 2.0, 40
    s, p, _ = surface_sim(b, fill=0.0, res=resolution, radius_m=radius_m)
    assert s.counts()[1] == 0
    dx = F(F(radius_m) / F(resolution))
    m = s.fluid_material()
    s.set_fluid_material(float(F(p.slurry.density_kg_m3) * dx * dx), m.h, m.rest_density)
    k = np.arange(-20, 21)
    jj, ii = np.meshgrid(k, k, indexing="ij")
    x = np.stack([ii.reshape(-1).astype(F) * dx, jj.reshape(-1).astype(F) * dx], axis=1)
    s.set_fluid(x, np.zeros_like(x), np.zeros(len(x), F))
    field, phi_full = s.surface_field()
    assert phi_full > 0.0
    c = G // 2
    for dj in (-1, 0, 1):
        for di in (-1, 0, 1):
            v = field[c + dj, c + di]
            assert abs(v - phi_full) / phi_full < 0.1, (v, phi_full)
    return field, phi_full


# surface.rs:505-518 no_fluid_gives_no_surface
def no_fluid_gives_no_surface(b):
    s, _, _ = surface_sim(b, fill=0.0, res=20)
    flat = s.surface_flat()
    assert list(flat) == [0.0]
    assert unflatten_polygons(flat) == []


# surface.rs:521-575 a_settled_puddle_has_one_closed_contour_of_plausible_area
def settled_puddle(b):
    s, p, drum = surface_sim(b)
    settle(s, p, drum)
    polys = s.surface()
    assert len(polys) == 1, f"expected one puddle contour, got {len(polys)}"
    poly = polys[0]
    assert len(poly) >= 8
    area = shoelace_area(poly)
    expected = 0.2 * math.pi * 0.5 * 0.5
    assert abs(area - expected) / expected < 0.35, (area, expected)
    points_inside(polys)
    return s


# surface.rs:578-629 spinning_drum_keeps_flung_fluid_contour_inside_the_wall
def spinning_drum_contour_inside(b):
    s, p, _ = surface_sim(b)
    spin_up(s, p)
    polys = s.surface()
    assert polys, "expected at least one contour"
    points_inside(polys)
    total = sum(shoelace_area(q) for q in polys)
    dx = s.fluid_material().h / 2.0
    footprint = s.counts()[1] * dx * dx
    assert total > 0.1 * footprint, (total, footprint)
    return s


# surface.rs:632-715 compacted_clump_does_not_hide_the_thin_film_contour
def compacted_clump(b):
    s, p, _ = surface_sim(b)
    spin_up(s, p)
    baseline = s.surface()
    assert baseline, "thin film alone produced no contour"
    base_area = sum(shoelace_area(q) for q in baseline)
    f = s.fluid()
    spacing = F(F(s.fluid_material().h) * F(0.05))
    n_side = 6
    clump = np.array([[F(F(F(i) - F(n_side / 2.0)) * spacing), F(F(F(j) - F(n_side / 2.0)) * spacing)]
                      for j in range(n_side) for i in range(n_side)], F)
    s.set_fluid(np.concatenate([f["x"], clump]), np.concatenate([f["v"], np.zeros_like(clump)]),
                np.concatenate([f["dye"], np.zeros(len(clump), F)]))
    polys = s.surface()
    assert polys, "expected a contour with a compacted clump present"
    area = sum(shoelace_area(q) for q in polys)
    assert area > 0.5 * base_area, (area, base_area)
    points_inside(polys)
    return s


# surface.rs:718-748 lifters_never_appear_inside_the_extracted_contour
def lifters_outside_contour(b, sdf_world):
    """sdf_world(drum, x, y, angle) -> distance, from the oracle's Drum::sdf_world."""
    s, p, drum = surface_sim(b, lifter_count=4)
    settle(s, p, drum)
    polys = s.surface()
    for poly in polys:
        for x, y in poly:
            d = sdf_world(drum, float(x), float(y), 0.0)
            assert d >= -1e-4, (x, y, d)
    return s


# surface.rs:761-777 flatten_polygons_round_trips_counts_and_points, on the flattened layout
def flatten_round_trip():
    flat = np.array([2, 3, 0, 0, 1, 0, 1, 1, 2, -1, -1, -2, -2], F)
    polys = unflatten_polygons(flat)
    assert len(polys) == 2
    assert polys[0].tolist() == [[0, 0], [1, 0], [1, 1]]
    assert polys[1].tolist() == [[-1, -1], [-2, -2]]


def isolated_points(b, every=4):
    """Many small closed contours: particles on every `every`-th grid point inside the wall, with
    a splat radius below one cell, so each is a lone field peak ringed by four segments."""
    s, p, _ = surface_sim(b, fill=0.0, res=24)
    cell = F(F(2.0 * 0.5) / F(G - 1))
    pts = []
    for gj in range(2, G - 2, every):
        for gi in range(2, G - 2, every):
            x = F(F(-0.5) + F(F(gi) * cell))
            y = F(F(-0.5) + F(F(gj) * cell))
            if x * x + y * y < 0.45 * 0.45:
                pts.append((x, y))
    m = s.fluid_material()
    s.set_fluid_material(m.particle_mass, float(F(cell) * F(0.5)), m.rest_density)
    s.set_fluid(np.array(pts, F))
    return s, len(pts)


def fallback_threshold(b):
    """A particle mass so small that analytic_phi_full exceeds every grid value: no contour at the
    analytic threshold, so extraction retries at half the measured peak (surface.rs:256-271)."""
    s, p, drum = surface_sim(b)
    settle(s, p, drum, steps=20)
    m = s.fluid_material()
    s.set_fluid_material(m.particle_mass * 1e-3, m.h, m.rest_density)
    return s
