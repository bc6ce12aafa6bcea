"""Helpers shared by the oracle and device tests: building params, drums and states the way the
reference's unit tests do (their fixtures: still_drum, single_ball, media_defaults, ...)."""
from __future__ import annotations

import math

import numpy as np

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import Simulation


def params(backend, preset=None, **kw):
    """Params::default() with dotted-path overrides, e.g. params(b, **{"mill.diameter_m": 0.2})."""
    p = backend.params_default()
    if preset:
        p = backend.preset(p, preset)
    for k, v in kw.items():
        obj = p
        parts = k.split(".")
        for part in parts[:-1]:
            obj = getattr(obj, part)
        setattr(obj, parts[-1], v)
    return p


def still_drum(radius, omega=0.0, lifters=None):
    """coupling.rs:130-139 / pbf.rs:2395-2404 / dem.rs still_drum"""
    d = capi.Drum()
    d.radius_m = radius
    d.omega = omega
    if lifters is not None:
        d.lifters = lifters
    return d


def lifters(count, height=0.02, base=0.03, top=0.02, phase=0.0):
    l = capi.LiftersParams()
    l.count, l.height_m, l.base_width_m, l.top_width_m, l.phase_deg = count, height, base, top, phase
    return l


def ball_mass(d, rho):
    """dem.rs:230-233 (f32 arithmetic)"""
    r = np.float32(d) * np.float32(0.5)
    return float(np.float32(rho) * np.float32(math.pi) * r * r)


def ball_inertia(m, r):
    """dem.rs:237-239"""
    return float(np.float32(0.5) * np.float32(m) * np.float32(r) * np.float32(r))


def empty_sim(backend, **kw):
    """A simulation with no balls and no fluid, ready for hand-built states."""
    p = params(backend, **{"slurry.enabled": 0, "media.fill_fraction": 0.0, **kw})
    s = Simulation(backend, p)
    s.set_balls(np.zeros((0, 2), np.float32))
    s.set_fluid(np.zeros((0, 2), np.float32))
    return s


def dem_state(backend, x, v, radius, mass, inertia=None, true_radius=None, theta=None, omega=None):
    """DemState { balls: Balls { ... } } built by hand (dem.rs tests)."""
    s = empty_sim(backend)
    x = np.asarray(x, np.float32).reshape(-1, 2)
    v = np.asarray(v, np.float32).reshape(-1, 2)
    s.set_balls(x, v, theta, omega)
    s.set_ball_material(radius, mass, ball_inertia(mass, radius) if inertia is None else inertia,
                        radius if true_radius is None else true_radius)
    return s


def media_defaults(backend):
    return backend.params_default().media.copy()


def slurry_defaults(backend):
    return backend.params_default().slurry.copy()
