"""Oracle pins against the reference's own unit tests: params.rs, rng.rs, grid.rs, geometry.rs and
the dem.rs scalar helpers. Each test names the reference test it restates."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

from milldynamics3_b200 import capi
from milldynamics3_b200.sim import MillError, probe_candidate_pairs, probe_grid, probe_neighbor_lists

from helpers import lifters, params, still_drum

F = np.float32


# ------------------------------------------------------------------ params.rs tests (:750-1203)
def test_default_params_are_valid(oracle):
    oracle.validate(oracle.params_default())


def test_critical_speed_matches_known_value(oracle):
    d = oracle.derived(params(oracle, **{"mill.diameter_m": 0.6}))
    assert abs(d.critical_speed_rpm - 54.61) < 0.1


def test_percent_critical_round_trips_through_rpm(oracle):
    p = params(oracle, **{"mill.speed_mode": capi.SPEED_PERCENT_CRITICAL, "mill.speed_value": 70.0})
    rpm = oracle.derived(p).rpm
    q = params(oracle, **{"mill.speed_mode": capi.SPEED_RPM, "mill.speed_value": rpm})
    assert abs(oracle.derived(q).percent_critical - 70.0) < 1e-3


def test_clockwise_direction_negates_omega(oracle):
    ccw = oracle.derived(params(oracle)).omega
    cw = oracle.derived(params(oracle, **{"mill.direction": capi.DIR_CW})).omega
    assert abs(ccw + cw) < 1e-6 and ccw > 0.0


@pytest.mark.parametrize("field,value", [("mill.diameter_m", 0.0), ("media.fill_fraction", 1.5),
                                         ("simulation.coarse_graining_k", 0.5),
                                         ("media.friction_ball_ball_static", 0.1)])
def test_invalid_params_rejected(oracle, field, value):
    with pytest.raises(MillError):
        oracle.validate(params(oracle, **{field: value}))


def test_zero_lifters_needs_no_geometry_bounds(oracle):
    oracle.validate(params(oracle, **{"lifters.count": 0, "lifters.height_m": 0.0, "lifters.base_width_m": 0.0,
                                      "lifters.top_width_m": 0.0}))


def test_effective_media_is_unscaled_when_true_count_is_small(oracle):
    p = params(oracle, **{"mill.diameter_m": 1.0, "media.ball_diameter_m": 0.3, "media.fill_fraction": 0.30,
                          "simulation.max_balls": 2000, "simulation.coarse_graining_mode": capi.CG_AUTO})
    d = oracle.derived(p)
    assert abs(d.eff_scale_factor - 1.0) < 1e-6 and abs(d.eff_diameter_m - d.eff_true_diameter_m) < 1e-6
    assert d.eff_ball_count < 2000


def test_effective_media_coarse_grains_when_true_count_is_large(oracle):
    p = params(oracle, **{"mill.diameter_m": 1.0, "mill.speed_value": 30.0, "media.ball_diameter_m": 0.010,
                          "simulation.coarse_graining_mode": capi.CG_AUTO})
    d = oracle.derived(p)
    assert d.true_ball_count > 600
    assert d.eff_scale_factor > 1.0 and d.eff_diameter_m > d.eff_true_diameter_m
    assert 300 < d.eff_ball_count <= 600


def test_coarse_graining_off_ignores_max_balls(oracle):
    p = params(oracle, **{"mill.diameter_m": 1.0, "mill.speed_value": 30.0, "media.ball_diameter_m": 0.010,
                          "simulation.coarse_graining_mode": capi.CG_OFF})
    d = oracle.derived(p)
    assert d.eff_scale_factor == 1.0 and d.eff_ball_count > 600
    assert d.eff_ball_count == int(np.round(F(d.true_ball_count)))


def test_coarse_graining_manual_uses_given_k(oracle):
    p = params(oracle, **{"media.ball_diameter_m": 0.3, "media.fill_fraction": 0.30, "simulation.max_balls": 2000,
                          "simulation.coarse_graining_mode": capi.CG_MANUAL, "simulation.coarse_graining_k": 2.0})
    oracle.validate(p)
    d = oracle.derived(p)
    assert abs(d.eff_scale_factor - 2.0) < 1e-6 and abs(d.eff_diameter_m - 2 * d.eff_true_diameter_m) < 1e-6


def test_shipped_defaults_need_no_coarse_graining_and_count_407(oracle):
    p = params(oracle, **{"simulation.coarse_graining_mode": capi.CG_AUTO})
    d = oracle.derived(p)
    assert d.true_ball_count <= 600 and d.eff_scale_factor == 1.0
    # The realtime preset: 407 ZrO2 discs (true count J*phi*R^2/r^2 rounded), 24 sub-steps.
    rt = oracle.derived(params(oracle, preset="realtime"))
    assert rt.eff_ball_count == 407 and rt.effective_substeps == 24 and rt.effective_fluid_resolution == 25


def test_effective_substeps_density_factor(oracle):
    # params.rs:705-726 doc: J = 0.30 -> 16, 0.40 -> 20, 0.50 -> 24 at the 2 mm / 63 mm default.
    for j, n in [(0.30, 16), (0.40, 20), (0.50, 24)]:
        assert oracle.derived(params(oracle, **{"media.fill_fraction": j})).effective_substeps == n


def test_presets(oracle):
    p = oracle.preset(oracle.params_default(), "impact_stats")
    assert p.simulation.substeps == 32 and p.simulation.dem_iterations == 12
    with pytest.raises(MillError):
        oracle.preset(oracle.params_default(), "nope")


# ------------------------------------------------------------------ rng.rs tests (:50-77)
def test_rng_deterministic_and_zero_seed_remapped(oracle_lib):
    s1 = C.c_uint64(oracle_lib.rng_seed_state(42))
    s2 = C.c_uint64(oracle_lib.rng_seed_state(42))
    for _ in range(100):
        assert oracle_lib.rng_next_u64(C.byref(s1)) == oracle_lib.rng_next_u64(C.byref(s2))
    z = C.c_uint64(oracle_lib.rng_seed_state(0))
    assert oracle_lib.rng_next_u64(C.byref(z)) != 0
    s = C.c_uint64(oracle_lib.rng_seed_state(7))
    for _ in range(1000):
        assert 0.0 <= oracle_lib.rng_next_f32(C.byref(s)) < 1.0


def test_rng_matches_xorshift64_star_restated_in_python(oracle_lib):
    state = 1
    s = C.c_uint64(oracle_lib.rng_seed_state(1))
    for _ in range(50):
        x = state
        x ^= (x << 13) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 7
        x ^= (x << 17) & 0xFFFFFFFFFFFFFFFF
        state = x
        assert oracle_lib.rng_next_u64(C.byref(s)) == (x * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF


# ------------------------------------------------------------------ grid.rs tests (:407-617)
def test_finds_all_pairs_within_cell_size_no_duplicates_no_self_pairs(oracle_lib):
    pts = [(0.0, 0.0), (0.05, 0.0), (0.0, 0.05), (100.0, 100.0)]
    rc, pairs = probe_candidate_pairs(oracle_lib, pts, 0.2)
    assert rc == 0
    pl = [tuple(p) for p in pairs]
    assert all(i < j for i, j in pl) and len(set(pl)) == len(pl)
    for e in [(0, 1), (0, 2), (1, 2)]:
        assert e in pl
    assert not any(3 in p for p in pl)


def test_candidate_pairs_are_a_superset_of_true_neighbours(oracle_lib):
    t = np.arange(40, dtype=np.float32) * F(0.37)
    pts = np.stack([np.sin(t) * 3, np.cos(t * F(1.3)) * 3], 1).astype(np.float32)
    _, pairs = probe_candidate_pairs(oracle_lib, pts, 1.0)
    cand = {tuple(p) for p in pairs}
    for i in range(40):
        for j in range(i + 1, 40):
            if np.linalg.norm(pts[i] - pts[j]) <= 1.0:
                assert (i, j) in cand


def test_for_each_near_finds_points_in_adjacent_cells(oracle_lib):
    pts = np.array([(0.9, 0.0), (-0.9, 0.0), (50.0, 50.0)], np.float32).reshape(-1)
    out = (C.c_uint32 * 16)()
    n = C.c_uint32()
    oracle_lib.probe_near(pts.ctypes.data_as(capi.f32p), 3, 1.0, 0.0, 0.0, out, 16, C.byref(n))
    assert sorted(out[k] for k in range(n.value)) == [0, 1]
    for p in [(math.inf, math.inf), (-math.inf, -math.inf), (math.inf, 0.0), (math.nan, math.nan)]:
        oracle_lib.probe_near(pts.ctypes.data_as(capi.f32p), 2, 1.0, p[0], p[1], out, 16, C.byref(n))
        assert n.value == 0


def test_empty_grid_has_no_pairs(oracle_lib):
    rc, pairs = probe_candidate_pairs(oracle_lib, np.zeros((0, 2), np.float32), 1.0)
    assert rc == 0 and len(pairs) == 0


def test_build_and_candidate_pairs_with_a_non_finite_point(oracle_lib):
    pts = [(0.0, 0.0), (0.05, 0.0), (math.inf, math.inf)]
    _, pairs = probe_candidate_pairs(oracle_lib, pts, 0.2)
    pl = [tuple(p) for p in pairs]
    assert (0, 1) in pl and not any(2 in p for p in pl)


def test_candidate_pair_order_is_deterministic_across_rebuilds(oracle_lib):
    t = np.arange(60, dtype=np.float32) * F(0.53)
    pts = np.stack([np.sin(t) * 2, np.cos(t * F(0.7)) * 2], 1)
    first = probe_candidate_pairs(oracle_lib, pts, 0.3)[1]
    for _ in range(5):
        assert np.array_equal(probe_candidate_pairs(oracle_lib, pts, 0.3)[1], first)


def test_sparse_fallback_matches_dense_layout_pair_order_and_set(oracle_lib):
    t = np.arange(20, dtype=np.float32) * F(0.41)
    pts = np.stack([np.sin(t) * F(0.5), np.cos(t * F(0.9)) * F(0.5)], 1)
    sp_pts = np.concatenate([pts, np.array([[1e6, 1e6]], np.float32)])
    rc, g = probe_grid(oracle_lib, sp_pts, 0.2)
    assert g["dense"] == 0
    rc, g2 = probe_grid(oracle_lib, pts, 0.2)
    assert g2["dense"] == 1
    assert np.array_equal(probe_candidate_pairs(oracle_lib, sp_pts, 0.2)[1],
                          probe_candidate_pairs(oracle_lib, pts, 0.2)[1])


def test_neighbor_lists_follow_the_fixed_stencil_order(oracle_lib):
    """pbf.rs:262-288: per-particle neighbour order is the 9-cell stencil order
    (-1,-1),(-1,0),(0,-1),(0,0),(+1,0),(+1,+1),(0,+1),(-1,+1),(+1,-1) relative to the particle's
    cell, ascending index within a cell -- restated here independently in Python."""
    rng = np.random.default_rng(3)
    pts = rng.uniform(-0.02, 0.02, size=(300, 2)).astype(np.float32)
    h = F(0.004)
    rc, off, nbrs = probe_neighbor_lists(oracle_lib, pts, float(h))
    keys = np.floor(pts / h).astype(np.int64)
    order = [(-1, -1), (-1, 0), (0, -1), (0, 0), (1, 0), (1, 1), (0, 1), (-1, 1), (1, -1)]
    for i in range(len(pts)):
        exp = []
        for dx, dy in order:
            cell = keys[i] + (dx, dy)
            for j in range(len(pts)):
                if j != i and keys[j][0] == cell[0] and keys[j][1] == cell[1]:
                    d = pts[i] - pts[j]
                    if F(d[0] * d[0]) + F(d[1] * d[1]) <= F(h * h):
                        exp.append(j)
        assert list(nbrs[off[i]:off[i + 1]]) == exp, i


# ------------------------------------------------------------------ geometry.rs tests (:294-527)
def sdfw(lib, drum, p, angle):
    d, nx, ny = C.c_float(), C.c_float(), C.c_float()
    lib.sdf_world(C.byref(drum), F(p[0]), F(p[1]), F(angle), C.byref(d), C.byref(nx), C.byref(ny))
    return d.value, np.array([nx.value, ny.value])


def toi(lib, drum, x0, x1, a0, a1, r):
    t = C.c_float()
    ok = lib.toi_swept(C.byref(drum), x0[0], x0[1], x1[0], x1[1], a0, a1, r, C.byref(t))
    return t.value if ok else None


def test_sdf_zero_at_wall_positive_inside(oracle_lib):
    d = still_drum(0.3)
    assert abs(oracle_lib.sdf_local(C.byref(d), 0.3, 0.0)) < 1e-6
    assert oracle_lib.sdf_local(C.byref(d), 0.0, 0.0) > 0 and oracle_lib.sdf_local(C.byref(d), 0.35, 0.0) < 0


def test_normal_points_inward_and_rotation_invariance(oracle_lib):
    d = still_drum(0.3)
    assert sdfw(oracle_lib, d, (0.3, 0.0), 0.0)[1][0] < -0.9
    p = np.array([0.25, 0.1], np.float32)
    d0 = sdfw(oracle_lib, d, p, 0.0)[0]
    a = 0.7
    pr = (p[0] * math.cos(a) - p[1] * math.sin(a), p[0] * math.sin(a) + p[1] * math.cos(a))
    assert abs(d0 - sdfw(oracle_lib, d, pr, a)[0]) < 1e-4
    n0 = sdfw(oracle_lib, d, (0.3, 0.0), 0.0)[1]
    n1 = sdfw(oracle_lib, d, (0.3, 0.0), 2 * math.pi)[1]
    assert np.linalg.norm(n0 - n1) < 1e-3


def test_sdf_world_never_manufactures_a_non_finite_result(oracle_lib):
    d = still_drum(0.3)
    for p in [(math.nan, 0.0), (math.inf, math.inf), (0.0, -math.inf)]:
        dd, n = sdfw(oracle_lib, d, p, 0.3)
        assert math.isfinite(dd) and np.all(np.isfinite(n)) and np.all(np.isfinite(-dd * n))


def test_lifters(oracle_lib):
    plain = still_drum(0.4)
    off = still_drum(0.4, lifters=lifters(0, 0.05, 0.05, 0.03, 12.0))
    for i in range(64):
        a = i * 2 * math.pi / 64
        assert abs(oracle_lib.sdf_local(C.byref(off), 0.4 * math.cos(a), 0.4 * math.sin(a)) -
                   oracle_lib.sdf_local(C.byref(plain), 0.4 * math.cos(a), 0.4 * math.sin(a))) < 1e-6
    ld = still_drum(0.3, lifters=lifters(8))
    assert oracle_lib.sdf_local(C.byref(ld), 0.29, 0.0) < 0.0
    a = 2 * math.pi / 16
    assert oracle_lib.sdf_local(C.byref(ld), 0.29 * math.cos(a), 0.29 * math.sin(a)) > 0.0
    one = still_drum(0.3, lifters=lifters(1))
    true_dist = math.hypot(0.27 - 0.28, 0.02 - 0.01)
    assert abs(sdfw(oracle_lib, one, (0.27, 0.02), 0.0)[0] - true_dist) < 1e-4
    tip = 0.3 - 0.02
    dd, n = sdfw(oracle_lib, ld, (tip - 0.005, 0.0), 0.0)
    assert dd > 0.0 and n[0] < -0.5


def test_wall_velocity_and_toi(oracle_lib):
    d = still_drum(0.3)
    t = toi(oracle_lib, d, (0.0, 0.0), (0.5, 0.0), 0.0, 0.0, 0.01)
    assert t is not None and abs(t - (0.3 - 0.01) / 0.5) < 1e-3
    x0 = float(F(0.3) - F(0.01))  # exactly touching, in f32 as the reference computes it
    assert toi(oracle_lib, d, (x0, 0.0), (float(F(x0) + F(0.001)), 0.0), 0.0, 0.0, 0.01) is None
    assert toi(oracle_lib, d, (0.0, 0.0), (0.01, 0.0), 0.0, 0.0, 0.01) is None
    one = still_drum(0.3, lifters=lifters(1))
    assert sdfw(oracle_lib, one, (0.29, 0.0), -0.3)[0] - 0.002 > 0.0
    assert toi(oracle_lib, one, (0.29, 0.0), (0.29, 0.0), -0.3, 0.0, 0.002) is not None


# ------------------------------------------------------------------ dem.rs helper tests (:1092-1121)
def test_effective_friction(oracle_lib):
    for vt in [-10.0, -0.02, 0.0, 0.001, 5.0]:
        assert oracle_lib.effective_friction(0.35, 0.35, vt, 0.02) == F(0.35)
    mk, ms, vs = 0.35, 1.2, 0.02
    f = lambda v: oracle_lib.effective_friction(mk, ms, v, vs)  # noqa: E731
    assert f(0.0) == F(ms) and f(0.05) == f(-0.05)
    assert F(ms) > f(0.01) > f(0.05) > f(1.0) and abs(f(1.0) - mk) < 1e-6


def test_impact_energy_bins(oracle_lib):
    assert oracle_lib.impact_energy_bin(0.0) == -1 and oracle_lib.impact_energy_bin(math.nan) == -1
    assert oracle_lib.impact_energy_bin(1e-9) == 0 and oracle_lib.impact_energy_bin(10.0) == 11
    assert oracle_lib.se_bin(1e-5) == 0 and oracle_lib.se_bin(1e9) == 27
