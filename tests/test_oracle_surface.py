"""surface::extract_surface on the oracle (surface.rs:233-430): the reference's own surface tests
(surface.rs:437-777), restated over the C ABI, plus structural checks of the flattened output."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from milldynamics3_b200 import capi

import surface_scenarios as sc


def _sdf_world(oracle_lib):
    def f(drum, x, y, angle):
        d, nx, ny = C.c_float(), C.c_float(), C.c_float()
        oracle_lib.sdf_world(C.byref(drum), x, y, angle, C.byref(d), C.byref(nx), C.byref(ny))
        return d.value
    return f


def test_splat_kernel_is_zero_outside_radius_and_positive_inside(oracle):
    sc.splat_kernel_zero_outside_radius(oracle)


def test_build_field_interior_value_matches_analytic_phi_full(oracle):
    sc.interior_value_matches_phi_full(oracle)


def test_no_fluid_gives_no_surface(oracle):
    sc.no_fluid_gives_no_surface(oracle)


def test_a_settled_puddle_has_one_closed_contour_of_plausible_area(oracle):
    sc.settled_puddle(oracle)


def test_spinning_drum_keeps_flung_fluid_contour_inside_the_wall(oracle):
    sc.spinning_drum_contour_inside(oracle)


def test_compacted_clump_does_not_hide_the_thin_film_contour(oracle):
    sc.compacted_clump(oracle)


def test_lifters_never_appear_inside_the_extracted_contour(oracle, oracle_lib):
    sc.lifters_outside_contour(oracle, _sdf_world(oracle_lib))


def test_flatten_polygons_round_trips_counts_and_points():
    sc.flatten_round_trip()


@pytest.mark.parametrize("every", [4, 2])
def test_isolated_points_give_one_smoothed_diamond_each(oracle, every):
    s, n = sc.isolated_points(oracle, every)
    polys = s.surface()
    assert len(polys) == n
    # four crossing edges around each peak, Chaikin-doubled
    assert all(len(q) == 8 for q in polys)


def test_fallback_threshold_finds_the_measured_peak_contour(oracle):
    s = sc.fallback_threshold(oracle)
    field, phi = s.surface_field()
    assert field.max() < 0.5 * phi
    polys = s.surface()
    assert polys
    sc.points_inside(polys)


def test_flattened_length_query(oracle):
    s = sc.settled_puddle(oracle)
    flat = s.surface_flat()
    n = C.c_uint32(0)
    assert s.lib.fluid_surface(s.h, None, 0, C.byref(n)) == 0 and n.value == len(flat)
    buf = np.zeros(len(flat) - 1, np.float32)
    rc = s.lib.fluid_surface(s.h, buf.ctypes.data_as(C.POINTER(C.c_float)), len(buf), C.byref(n))
    assert rc == capi.MG_ERR_CAPACITY
    assert int(flat[0]) == 1 and int(flat[1]) * 2 + 2 == len(flat)
