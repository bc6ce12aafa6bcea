"""The benchmark's mills, built through the C ABI's Params (the reference's Params::default() plus
overrides, params.rs:62-77 and following), one builder per configuration:

* realtime: the 'realtime' preset exactly as Params supplies it (63 mm drum, 407 discs of 2 mm,
  794 fluid particles at resolution 25, 24 sub-steps per frame);
* realtime_300: the same mill with 300 steel discs (7800 kg/m^3) placed uniformly at random
  without overlap in the lower drum (Simulation::with_initial_balls, lib.rs:138-204). The lower
  half alone would need a packing of 0.65, past what random placement reaches (~0.55), so the
  discs fill the part of the drum below 0.35 R (packing 0.45);
* dem_only(n): balls only (slurry off), monodisperse discs of 5 mm radius (the reference supports
  one radius per population, dem.rs:275-276), 7800 kg/m^3, friction 0.3 (kinetic and static,
  ball-ball and ball-wall), restitution 0.5, 30 % fill at 60 % of critical speed; the drum is
  scaled to hold n discs, D = 2 r sqrt(n / (J phi)) (0.45 m for 500, 0.90 m for 2,000, 2.85 m
  for 20,000, 9.02 m for 200,000: 200,000 discs of 5 mm do not fit in a 1 m drum);
* large(resolution, viscosity): 5,000 discs of 2 mm in a 221 mm drum (5,000 discs of 2 mm do not
  fit in the 63 mm drum; D = 2 r sqrt(5000 / (J phi)) at the default J = 0.5 holds 5,006) with
  the fluid at resolution 100 (~12.7k particles) or 200 (~50.8k), viscosity 1e-3 or 1e-1 Pa s.

The batched and served mills (the 512-mill mix) are drawn by batch.mix_params.
"""
from __future__ import annotations

import math

import numpy as np

from . import capi


def _set(p, path, value):
    obj = p
    parts = path.split(".")
    for part in parts[:-1]:
        obj = getattr(obj, part)
    setattr(obj, parts[-1], value)


def realtime(b):
    return b.preset(b.params_default(), "realtime"), None


def lower_drum_discs(n, drum_radius, ball_radius, seed, top=0.35):
    """n non-overlapping disc centres drawn uniformly (rejection sampling) in the drum below
    y = top * R, one radius clear of the wall; float32, shape (n, 2)."""
    rng = np.random.default_rng(seed)
    rmax = drum_radius - 1.05 * ball_radius
    pts = np.zeros((0, 2))
    min2 = (2.02 * ball_radius) ** 2
    while len(pts) < n:
        x, y = rng.uniform(-rmax, rmax), rng.uniform(-rmax, top * rmax)
        if x * x + y * y > rmax * rmax:
            continue
        if len(pts) and (((pts - (x, y)) ** 2).sum(axis=1) < min2).any():
            continue
        pts = np.vstack([pts, (x, y)])
    return pts.astype(np.float32)


def realtime_300(b):
    p = b.preset(b.params_default(), "realtime")
    _set(p, "media.density_kg_m3", 7800.0)
    return p, lower_drum_discs(300, 0.0315, 0.001, seed=2024)


DEM_FILL = 0.3


def dem_only_params(p, n_balls=None, diameter_m=None):
    """The DEM-only configuration for n_balls discs (drum scaled to hold them) or for a given
    drum diameter."""
    phi = float(p.media.packing_fraction_2d)
    r = 0.005
    if diameter_m is None:
        diameter_m = 2.0 * r * math.sqrt(n_balls / (DEM_FILL * phi))
    for k, v in {"slurry.enabled": 0, "mill.diameter_m": diameter_m, "mill.speed_mode": capi.SPEED_PERCENT_CRITICAL,
                 "mill.speed_value": 60.0, "media.fill_fraction": DEM_FILL, "media.ball_diameter_m": 2 * r,
                 "media.density_kg_m3": 7800.0, "media.friction_ball_ball": 0.3, "media.friction_ball_wall": 0.3,
                 "media.friction_ball_ball_static": 0.3, "media.friction_ball_wall_static": 0.3,
                 "media.restitution_ball_ball": 0.5, "media.restitution_ball_wall": 0.5}.items():
        _set(p, k, v)
    return p


def dem_only(b, n_balls):
    p = dem_only_params(b.params_default(), n_balls)
    b.validate(p)
    return p, None


def large_params(p, resolution, viscosity):
    for k, v in {"mill.diameter_m": 0.221, "media.ball_diameter_m": 0.002, "simulation.resolution": resolution,
                 "slurry.viscosity_pa_s": viscosity}.items():
        _set(p, k, v)
    return p


def large(b, resolution=100, viscosity=1e-3):
    p = large_params(b.params_default(), resolution, viscosity)
    b.validate(p)
    return p, None
