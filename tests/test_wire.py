"""The JSON wire format of the reference's WASM binding (milldynamics3_b200.wire): serde's Params
representation in and out, Simulation::metrics and SeedResult out."""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np
import pytest

from milldynamics3_b200 import capi, wire
from milldynamics3_b200.sim import Simulation

HERE = os.path.dirname(os.path.abspath(__file__))


def _bytes(p):
    return bytes(C.string_at(C.addressof(p), C.sizeof(p)))


def test_params_round_trip(oracle):
    for preset in (None, "realtime"):
        p = oracle.params_default() if preset is None else oracle.preset(oracle.params_default(), preset)
        text = wire.params_to_json(p)
        q = wire.params_from_json(text)
        assert _bytes(q) == _bytes(p)
        assert wire.params_to_json(q) == text


def test_params_json_layout(oracle):
    d = json.loads(wire.params_to_json(oracle.params_default()))
    assert list(d) == ["mill", "media", "slurry", "lifters", "simulation"]
    assert d["mill"]["speed_mode"] in ("rpm", "percent_critical")
    assert d["slurry"]["enabled"] in (True, False)
    assert isinstance(d["simulation"]["seed"], int) and isinstance(d["lifters"]["count"], int)
    assert d["simulation"]["coarse_graining_mode"] == "off"


def test_every_field_and_option_the_web_client_sends(oracle):
    schema = json.load(open(os.path.join(HERE, "golden", "wire_schema.json")))
    base = json.loads(wire.params_to_json(oracle.params_default()))
    for f in schema["fields"]:
        sec, name = f["path"].split(".")
        assert name in base[sec], f["path"]
        for opt in f["options"]:
            doc = json.loads(json.dumps(base))
            doc[sec][name] = opt
            p = wire.params_from_json(doc)
            assert json.loads(wire.params_to_json(p))[sec][name] == opt


def test_serde_defaults_and_required_fields(oracle):
    base = json.loads(wire.params_to_json(oracle.params_default()))
    older = json.loads(json.dumps(base))
    for sec, name in [("media", "friction_ball_ball_static"), ("media", "friction_ball_wall_static"),
                      ("media", "friction_velocity_scale_m_s"), ("slurry", "surface_tension_n_m")]:
        del older[sec][name]
    p = wire.params_from_json(older)
    assert p.media.friction_ball_ball_static == np.float32(0.25)
    assert p.media.friction_ball_wall_static == np.float32(0.35)
    assert p.media.friction_velocity_scale_m_s == np.float32(0.02)
    assert p.slurry.surface_tension_n_m == np.float32(0.072)
    for sec, name in [("mill", "diameter_m"), ("slurry", "rheology"), ("simulation", "seed")]:
        doc = json.loads(json.dumps(base))
        del doc[sec][name]
        with pytest.raises(wire.WireError, match=name):
            wire.params_from_json(doc)
    doc = json.loads(json.dumps(base))
    doc["mill"]["unknown_field"] = 3      # serde ignores unknown fields
    wire.params_from_json(doc)


@pytest.mark.parametrize("sec,name,value", [("slurry", "enabled", 1), ("lifters", "count", 1.5),
                                            ("lifters", "count", -1), ("mill", "speed_mode", "fast"),
                                            ("mill", "diameter_m", "1.0"), ("simulation", "seed", True)])
def test_wrong_types_are_rejected(oracle, sec, name, value):
    doc = json.loads(wire.params_to_json(oracle.params_default()))
    doc[sec][name] = value
    with pytest.raises(wire.WireError, match=name):
        wire.params_from_json(doc)


def test_f32_numbers_are_shortest_and_exact(oracle):
    p = oracle.params_default()
    p.mill.diameter_m = 0.1
    p.media.density_kg_m3 = 7850.0
    p.lifters.height_m = 1e-7
    d = wire.params_to_json(p)
    assert '"diameter_m":0.1,' in d and '"density_kg_m3":7850.0,' in d
    assert '"height_m":1e-7,' in d
    assert _bytes(wire.params_from_json(d)) == _bytes(p)


@pytest.mark.parametrize("value,kind,text", [
    (1e-7, "f32", "1e-7"), (2.5e20, "f32", "2.5e20"), (1e-6, "f32", "0.000001"), (1e13, "f32", "1e13"),
    (1.5e12, "f32", "1500000000000.0"), (-0.0, "f32", "-0.0"), (0.072, "f32", "0.072"), (3.0, "f32", "3.0"),
    (1e-5, "f64", "0.00001"), (2.5e-7, "f64", "2.5e-7"), (1e16, "f64", "1e16"), (1e15, "f64", "1000000000000000.0"),
    (1.7976931348623157e308, "f64", "1.7976931348623157e308"), (5e-324, "f64", "5e-324")])
def test_numbers_are_written_as_serde_json_writes_them(value, kind, text):
    # serde_json prints floats with the ryu crate: shortest digits, plain notation in a window of
    # exponents, otherwise mantissa 'e' exponent with no '+' and no leading zeros
    assert wire._num(value, kind).text == text


def test_metrics_json_has_the_metrics_struct_fields(oracle):
    s = Simulation(oracle, oracle.preset(oracle.params_default(), "realtime"))
    s.step(1.0 / 60.0)
    d = json.loads(wire.metrics_to_json(s))
    assert list(d) == [
        "toe_angle_rad", "shoulder_angle_rad", "charge_centroid_m", "pool_angle_min_rad", "pool_angle_max_rad",
        "free_surface_angle_rad", "free_surface_offset_m", "pool_depth_m", "mixing_index", "total_kinetic_energy_j",
        "max_ball_overlap_fraction", "max_ball_wall_overlap_fraction", "max_fluid_density_error_fraction",
        "drum_omega_rad_s", "fluid_particle_count", "mean_fluid_density_error_fraction",
        "max_fluid_compression_error_fraction", "mean_fluid_compression_error_fraction", "power_draw_w",
        "torque_nm", "collision_rate_per_s", "dissipated_power_w", "impact_energy_histogram", "stress",
        "coupling_clamp_hits", "effective_ball_diameter_m", "simulated_ball_count", "true_ball_count",
        "coarse_graining_factor", "max_substep_displacement_over_diameter", "mean_shear_rate_per_s",
        "viscosity_solver_iterations"]
    m = s.metrics()
    assert len(d["charge_centroid_m"]) == 2
    assert np.float32(d["charge_centroid_m"][0]) == np.float32(m.charge_centroid_m[0])
    assert d["fluid_particle_count"] == s.counts()[1]
    assert len(d["impact_energy_histogram"]["bin_edges_j"]) == capi.SE_BINS + 1
    assert len(d["impact_energy_histogram"]["counts_per_s"]) == capi.SE_BINS
    assert len(d["stress"]["thresholds_scaled"]) == 6
    assert np.float32(d["power_draw_w"]) == np.float32(s.scalars().power_draw_w)
    if not m.valid & capi.METRIC_TOE_SHOULDER:
        assert d["toe_angle_rad"] is None


def test_seed_result_json(oracle):
    from milldynamics3_b200 import seeds
    p = oracle.params_default()
    p.slurry.enabled = 0
    p.simulation.max_balls = 60
    r = seeds.run_seed(oracle, p, 1, 0.0, 1.0)
    d = json.loads(wire.seed_result_to_json(r))
    assert list(d) == ["seed", "window_s", "coarse_graining_factor", "names", "values", "power_drift_rel_per_rev"]
    assert d["names"] == r.names and d["values"] == [v if np.isfinite(v) else None for v in r.values]
    c = json.loads(wire.combined_to_json(seeds.combine(oracle, [r, r])))
    assert c["seeds"] == 2 and c["std_err"] == [0.0] * len(r.values)
