"""The JSON wire format of the reference's WASM binding (crates/mill-wasm/src/lib.rs), so the
existing web frontend can talk to a GPU server.

* Params in and out: serde's representation of `Params` (params.rs:8-545): snake_case field
  names in declaration order, enums as snake_case strings, `slurry.enabled` a JSON bool, integers
  for the u32/u64 fields. As serde reads it, every field is required except the four with
  `#[serde(default = ...)]` (params.rs:162-175, 339-340), which take their default functions'
  values; unknown fields are ignored; a wrong type or a missing field is an error naming it.
* Metrics out: `Simulation::metrics` (lib.rs:370-412) serialised as `metrics_json` does
  (mill-wasm lib.rs:164-166): `metrics::Metrics` (metrics.rs:69-110) with `Option` as null, the
  centroid tuple as a two-element array, `stress` as `StressMetrics` (stress.rs:243-273) and the
  impact-energy histogram's bin edges and rates. serde_json writes non-finite floats as null.
* Seed results out: `batch::SeedResult` / `Combined` (batch.rs:13-34) as `stress_run_json`
  returns them (mill-wasm lib.rs:188-204).

Floats are written with the shortest digits that read back to the same f32 (or f64) value, so a
reader gets the same numbers as from serde_json.
"""
from __future__ import annotations

import json
import math

import numpy as np

from . import capi

F = np.float32

_ENUMS = {
    ("mill", "speed_mode"): ["rpm", "percent_critical"],
    ("mill", "direction"): ["counter_clockwise", "clockwise"],
    ("slurry", "rheology"): ["newtonian", "bingham"],
    ("slurry", "dye_pattern"): ["left_right", "top_bottom", "none"],
    ("simulation", "coarse_graining_mode"): ["auto", "off", "manual"],
}
# params.rs:53-60, 130-178, 300-342, 409-417, 449-484 (declaration order); kind per field
_FIELDS = {
    "mill": [("diameter_m", "f32"), ("speed_mode", "enum"), ("speed_value", "f32"), ("direction", "enum")],
    "media": [("ball_diameter_m", "f32"), ("fill_fraction", "f32"), ("packing_fraction_2d", "f32"),
              ("density_kg_m3", "f32"), ("restitution_ball_ball", "f32"), ("restitution_ball_wall", "f32"),
              ("friction_ball_ball", "f32"), ("friction_ball_wall", "f32"), ("friction_ball_ball_static", "f32"),
              ("friction_ball_wall_static", "f32"), ("friction_velocity_scale_m_s", "f32"),
              ("rolling_friction", "f32")],
    "slurry": [("enabled", "bool"), ("fill_fraction", "f32"), ("density_kg_m3", "f32"), ("viscosity_pa_s", "f32"),
               ("rheology", "enum"), ("yield_stress_pa", "f32"), ("wall_no_slip", "f32"), ("ball_no_slip", "f32"),
               ("wettability", "f32"), ("surface_tension_n_m", "f32"), ("dye_pattern", "enum")],
    "lifters": [("count", "u32"), ("height_m", "f32"), ("base_width_m", "f32"), ("top_width_m", "f32"),
                ("phase_deg", "f32")],
    "simulation": [("resolution", "u32"), ("substeps", "u32"), ("pbf_iterations", "u32"), ("dem_iterations", "u32"),
                   ("time_scale", "f32"), ("frame_budget_ms", "f32"), ("max_balls", "u32"), ("seed", "u64"),
                   ("coarse_graining_mode", "enum"), ("coarse_graining_k", "f32")],
}
_SECTIONS = ("mill", "media", "slurry", "lifters", "simulation")
# #[serde(default = "...")] fields and their default functions' values (params.rs:184-198, 347-349)
_SERDE_DEFAULTS = {
    ("media", "friction_ball_ball_static"): 0.25,
    ("media", "friction_ball_wall_static"): 0.35,
    ("media", "friction_velocity_scale_m_s"): 0.02,
    ("slurry", "surface_tension_n_m"): 0.072,
}


class WireError(ValueError):
    """A JSON document serde would reject (the message names the field)."""


class _Num:
    """A JSON number with its text chosen (shortest f32 or f64 digits)."""

    def __init__(self, text):
        self.text = text


def _ryu_text(v, f32: bool) -> str:
    """The text serde_json writes for a finite float (the ryu crate's format32 / format64): the
    shortest digits that read back to the same value, in plain notation when the decimal point
    falls within reach (10^-6 <= |v| < 10^13 for f32, 10^-5 <= |v| < 10^16 for f64, whole numbers
    with a trailing '.0'), else as d.ddd followed by 'e' and the exponent without '+' or leading
    zeros ('1e-7', '2.5e20')."""
    neg = bool(np.signbit(v))
    if v == 0:
        return "-0.0" if neg else "0.0"
    sci = np.format_float_scientific(abs(v), unique=True, trim="-")
    mant, ex = sci.split("e")
    digits = mant.replace(".", "")
    kk = int(ex) + 1  # 10^(kk-1) <= |v| < 10^kk
    n = len(digits)
    hi, lo = (13, -6) if f32 else (16, -5)
    if kk - n >= 0 and kk <= hi:
        t = digits + "0" * (kk - n) + ".0"
    elif 0 < kk <= hi:
        t = digits[:kk] + "." + digits[kk:]
    elif lo < kk <= 0:
        t = "0." + "0" * (-kk) + digits
    elif n == 1:
        t = digits + "e" + str(kk - 1)
    else:
        t = digits[0] + "." + digits[1:] + "e" + str(kk - 1)
    return "-" + t if neg else t


def _num(x, kind: str):
    if kind == "f32":
        v = F(x)
        return _Num(_ryu_text(v, True)) if np.isfinite(v) else None
    v = np.float64(x)
    return _Num(_ryu_text(v, False)) if np.isfinite(v) else None


def _dumps(obj) -> str:
    """Compact JSON in serde_json's layout; numbers keep the text _num chose."""
    if obj is None:
        return "null"
    if isinstance(obj, _Num):
        return obj.text
    if isinstance(obj, bool):
        return "true" if obj else "false"
    if isinstance(obj, int):
        return str(obj)
    if isinstance(obj, float):
        return _ryu_text(np.float64(obj), False) if math.isfinite(obj) else "null"
    if isinstance(obj, str):
        return json.dumps(obj)
    if isinstance(obj, dict):
        return "{" + ",".join(json.dumps(k) + ":" + _dumps(v) for k, v in obj.items()) + "}"
    return "[" + ",".join(_dumps(v) for v in obj) + "]"


def _read(section: str, name: str, kind: str, value):
    where = f"{section}.{name}"
    if kind == "f32":
        if isinstance(value, bool) or not isinstance(value, (int, float)):
            raise WireError(f"invalid type for `{where}`: expected f32")
        return float(F(float(value)))
    if kind in ("u32", "u64"):
        if isinstance(value, bool) or not isinstance(value, int):
            raise WireError(f"invalid type for `{where}`: expected {kind}")
        if value < 0 or value >= (1 << (32 if kind == "u32" else 64)):
            raise WireError(f"invalid value for `{where}`: out of range for {kind}")
        return value
    if kind == "bool":
        if not isinstance(value, bool):
            raise WireError(f"invalid type for `{where}`: expected a boolean")
        return 1 if value else 0
    names = _ENUMS[(section, name)]
    if not isinstance(value, str) or value not in names:
        raise WireError(f"unknown variant `{value}` for `{where}`, expected one of {', '.join(names)}")
    return names.index(value)


def params_from_json(doc) -> capi.Params:
    """serde_json::from_str::<Params> (mill-wasm lib.rs:25-45): a JSON text or an already parsed
    dict to capi.Params."""
    if isinstance(doc, (str, bytes)):
        try:
            doc = json.loads(doc)
        except json.JSONDecodeError as e:
            raise WireError(str(e)) from None
    if not isinstance(doc, dict):
        raise WireError("invalid type: expected struct Params")
    p = capi.Params()
    for sec in _SECTIONS:
        if sec not in doc:
            raise WireError(f"missing field `{sec}`")
        d = doc[sec]
        if not isinstance(d, dict):
            raise WireError(f"invalid type for `{sec}`: expected a struct")
        obj = getattr(p, sec)
        for name, kind in _FIELDS[sec]:
            if name in d:
                v = _read(sec, name, kind, d[name])
            elif (sec, name) in _SERDE_DEFAULTS:
                v = float(F(_SERDE_DEFAULTS[(sec, name)]))
            else:
                raise WireError(f"missing field `{name}` in `{sec}`")
            setattr(obj, name, v)
    return p


def params_to_dict(p: capi.Params) -> dict:
    out = {}
    for sec in _SECTIONS:
        obj = getattr(p, sec)
        d = {}
        for name, kind in _FIELDS[sec]:
            v = getattr(obj, name)
            if kind == "f32":
                d[name] = _num(v, "f32")
            elif kind == "bool":
                d[name] = bool(v)
            elif kind == "enum":
                d[name] = _ENUMS[(sec, name)][int(v)]
            else:
                d[name] = int(v)
        out[sec] = d
    return out


def params_to_json(p: capi.Params) -> str:
    """serde_json::to_string(&Params) (mill-wasm lib.rs:157-159, 172-174)."""
    return _dumps(params_to_dict(p))


def _opt(valid: int, bit: int, *vals):
    if not valid & bit:
        return None
    return _num(vals[0], "f32") if len(vals) == 1 else [_num(v, "f32") for v in vals]


def _round_half_away(x: float) -> float:
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def metrics_to_dict(sim) -> dict:
    """Simulation::metrics (lib.rs:370-412) of a milldynamics3_b200.sim.Simulation."""
    m = sim.metrics()
    sc = sim.scalars()
    st = sim.stress_metrics()
    rate = sim.stress_histogram_rate()
    d = sim.b.derived(sim.params)
    v = m.valid
    edges = [10.0 ** (-3.0 + i / 4.0) for i in range(capi.SE_BINS + 1)]   # stress.rs:28-55
    scale_j = float(st.scale_energy_j)

    def f32(x):
        return _num(x, "f32")

    def f64(x):
        return _num(x, "f64")
    return {
        "toe_angle_rad": _opt(v, capi.METRIC_TOE_SHOULDER, m.toe_angle_rad),
        "shoulder_angle_rad": _opt(v, capi.METRIC_TOE_SHOULDER, m.shoulder_angle_rad),
        "charge_centroid_m": _opt(v, capi.METRIC_CENTROID, *m.charge_centroid_m),
        "pool_angle_min_rad": _opt(v, capi.METRIC_POOL_EXTENT, m.pool_angle_min_rad),
        "pool_angle_max_rad": _opt(v, capi.METRIC_POOL_EXTENT, m.pool_angle_max_rad),
        "free_surface_angle_rad": _opt(v, capi.METRIC_FREE_SURFACE, m.free_surface_angle_rad),
        "free_surface_offset_m": _opt(v, capi.METRIC_FREE_SURFACE, m.free_surface_offset_m),
        "pool_depth_m": _opt(v, capi.METRIC_POOL_DEPTH, m.pool_depth_m),
        "mixing_index": _opt(v, capi.METRIC_MIXING, m.mixing_index),
        "total_kinetic_energy_j": f32(m.total_kinetic_energy_j),
        "max_ball_overlap_fraction": f32(m.max_ball_overlap_fraction),
        "max_ball_wall_overlap_fraction": f32(m.max_ball_wall_overlap_fraction),
        "max_fluid_density_error_fraction": _opt(v, capi.METRIC_DENSITY, m.max_fluid_density_error_fraction),
        "drum_omega_rad_s": f32(m.drum_omega_rad_s),
        "fluid_particle_count": int(m.fluid_particle_count),
        "mean_fluid_density_error_fraction": _opt(v, capi.METRIC_DENSITY, m.mean_fluid_density_error_fraction),
        "max_fluid_compression_error_fraction": _opt(v, capi.METRIC_DENSITY, m.max_fluid_compression_error_fraction),
        "mean_fluid_compression_error_fraction": _opt(v, capi.METRIC_DENSITY,
                                                      m.mean_fluid_compression_error_fraction),
        "power_draw_w": f32(sc.power_draw_w),
        "torque_nm": f32(sc.torque_nm),
        "collision_rate_per_s": f32(sc.collision_rate_per_s),
        "dissipated_power_w": f32(sc.dissipated_power_w),
        "impact_energy_histogram": {
            "bin_edges_j": [f32(e * scale_j) for e in edges],
            "counts_per_s": [f32(c) for c in rate],
        },
        "stress": {
            "ball_mass_3d_kg": f32(st.ball_mass_3d_kg),
            "scale_energy_j": f32(st.scale_energy_j),
            "impacts_per_ball_per_s": [f32(x) for x in st.impacts_per_ball_per_s],
            "impacts_total_per_ball_per_s": f32(st.impacts_total_per_ball_per_s),
            "mean_se_scaled": [f32(x) for x in st.mean_se_scaled],
            "mean_se_scaled_drop": f32(st.mean_se_scaled_drop),
            "mean_se_scaled_shear": f32(st.mean_se_scaled_shear),
            "stress_intensity_scaled": f32(st.stress_intensity_scaled),
            "wall_power_per_ball_w": f32(st.wall_power_per_ball_w),
            "specific_power_w_per_kg": f32(st.specific_power_w_per_kg),
            "thresholds_scaled": [f32(x) for x in st.thresholds_scaled],
            "effective_power_per_ball_w": [f32(x) for x in st.effective_power_per_ball_w],
            "cumulative_wall_energy_per_ball_j": f64(st.cumulative_wall_energy_per_ball_j),
            "cumulative_specific_energy_j_per_kg": f64(st.cumulative_specific_energy_j_per_kg),
            "cumulative_effective_energy_per_ball_j": [f64(x) for x in st.cumulative_effective_energy_per_ball_j],
        },
        "coupling_clamp_hits": int(sc.coupling_clamp_hits),
        "effective_ball_diameter_m": f32(d.eff_diameter_m),
        "simulated_ball_count": int(d.eff_ball_count),
        "true_ball_count": int(max(_round_half_away(float(F(d.true_ball_count))), 0.0)),
        "coarse_graining_factor": f32(d.eff_scale_factor),
        "max_substep_displacement_over_diameter": f32(sc.max_substep_displacement_over_diameter),
        "mean_shear_rate_per_s": f32(sc.mean_shear_rate_per_s),
        "viscosity_solver_iterations": int(sc.viscosity_iterations),
    }


def metrics_to_json(sim) -> str:
    """Simulation::metrics_json (mill-wasm lib.rs:164-166)."""
    return _dumps(metrics_to_dict(sim))


def seed_result_to_json(r) -> str:
    """batch::SeedResult (batch.rs:13-25) as stress_run_json returns it; r is a
    milldynamics3_b200.seeds.SeedResult."""
    return _dumps({"seed": int(r.seed), "window_s": _num(r.window_s, "f64"),
                   "coarse_graining_factor": _num(r.coarse_graining_factor, "f32"),
                   "names": list(r.names), "values": [_num(x, "f64") for x in r.values],
                   "power_drift_rel_per_rev": _num(r.power_drift_rel_per_rev, "f64")})


def combined_to_json(c) -> str:
    """batch::Combined (batch.rs:28-34)."""
    return _dumps({"names": list(c.names), "mean": [_num(x, "f64") for x in c.mean],
                   "std_err": [_num(x, "f64") for x in c.std_err], "seeds": int(c.seeds)})
