"""surface::extract_surface on the device (two kernel launches) gives exactly the oracle's
flattened polygons and occupancy field, and passes surface.rs's own tests."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from milldynamics3_b200.sim import Simulation

import surface_scenarios as sc

pytestmark = pytest.mark.gpu


def _same(ds, os_):
    dflat, oflat = ds.surface_flat(), os_.surface_flat()
    assert len(dflat) == len(oflat), (len(dflat), len(oflat))
    assert np.array_equal(dflat.view(np.uint32), oflat.view(np.uint32)), \
        int(np.flatnonzero(dflat.view(np.uint32) != oflat.view(np.uint32))[0])
    (df, dp), (of, op) = ds.surface_field(), os_.surface_field()
    assert np.array_equal(df.view(np.uint32), of.view(np.uint32))
    assert np.float32(dp).view(np.uint32) == np.float32(op).view(np.uint32)
    return dflat


def _preset(b, name):
    return b.params_default() if name == "default" else b.preset(b.params_default(), name)


@pytest.mark.parametrize("preset,frames", [("realtime", 0), ("realtime", 8), ("default", 3)])
def test_device_surface_matches_oracle_on_presets(device, oracle, preset, frames):
    sims = []
    for b in (device, oracle):
        s = Simulation(b, _preset(b, preset))
        for _ in range(frames):
            s.step(1.0 / 60.0)
        sims.append(s)
    assert sims[0].state_hash(True) == sims[1].state_hash(True)
    flat = _same(*sims)
    assert flat[0] >= 1


def test_device_surface_matches_oracle_with_lifters(device, oracle):
    sims = []
    for b in (device, oracle):
        p = b.params_default()
        p.lifters.count = 8
        p.lifters.height_m = 0.004
        p.lifters.base_width_m = 0.006
        p.lifters.top_width_m = 0.003
        b.validate(p)
        s = Simulation(b, p)
        for _ in range(4):
            s.step(1.0 / 60.0)
        sims.append(s)
    _same(*sims)


@pytest.mark.parametrize("case", ["settled_puddle", "spinning_drum_contour_inside", "compacted_clump",
                                  "no_fluid_gives_no_surface"])
def test_device_runs_reference_surface_tests_with_oracle_bits(device, oracle, case):
    ds = getattr(sc, case)(device)
    os_ = getattr(sc, case)(oracle)
    if ds is not None:
        _same(ds, os_)


def test_device_lifters_never_inside_contour(device, oracle, oracle_lib):
    def sdf_world(drum, x, y, angle):
        d, nx, ny = C.c_float(), C.c_float(), C.c_float()
        oracle_lib.sdf_world(C.byref(drum), x, y, angle, C.byref(d), C.byref(nx), C.byref(ny))
        return d.value
    _same(sc.lifters_outside_contour(device, sdf_world), sc.lifters_outside_contour(oracle, sdf_world))


def test_device_field_splat_and_interior_value(device, oracle):
    sc.splat_kernel_zero_outside_radius(device)
    df, dp = sc.interior_value_matches_phi_full(device)
    of, op = sc.interior_value_matches_phi_full(oracle)
    assert np.array_equal(df.view(np.uint32), of.view(np.uint32)) and dp == op


@pytest.mark.parametrize("every", [4, 2])
def test_device_many_isolated_contours(device, oracle, every):
    # every=2 gives ~9500 segments, more than the links kept in shared memory
    (ds, n), (os_, _) = sc.isolated_points(device, every), sc.isolated_points(oracle, every)
    flat = _same(ds, os_)
    assert int(flat[0]) == n
    assert every != 2 or 4 * n > 4096


def test_device_fallback_threshold(device, oracle):
    _same(sc.fallback_threshold(device), sc.fallback_threshold(oracle))


def test_device_nonfinite_particles(device, oracle):
    sims = []
    for b in (device, oracle):
        s, p, drum = sc.surface_sim(b)
        sc.settle(s, p, drum, steps=10)
        f = s.fluid()
        x = f["x"].copy()
        x[3] = (np.nan, 0.1)
        x[7] = (np.inf, -np.inf)
        s.set_fluid(x, f["v"], f["dye"])
        sims.append(s)
    _same(*sims)


def test_device_surface_repeatable(device):
    s = Simulation(device, _preset(device, "realtime"))
    s.step(1.0 / 60.0)
    a = s.surface_flat()
    b = s.surface_flat()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
