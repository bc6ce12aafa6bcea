"""ctypes mirror of include/millgpu.h.

`Lib(path, prefix)` binds every entry point of the header from a shared library under a name
prefix ("mg_" for the CUDA library). The structs below are field-for-field copies of the header,
which in turn mirrors the reference's Rust types (params.rs, pbf.rs, dem.rs, lib.rs).
"""
from __future__ import annotations

import ctypes as C

MG_OK = 0
MG_ERR_INVALID_PARAMS = 1
MG_ERR_ARG = 2
MG_ERR_CUDA = 3
MG_ERR_CAPACITY = 4
MG_ERR_NO_DEVICE = 5
MG_ERR_STATE = 6

SPEED_RPM, SPEED_PERCENT_CRITICAL = 0, 1
DIR_CCW, DIR_CW = 0, 1
CG_AUTO, CG_OFF, CG_MANUAL = 0, 1, 2
RHEOLOGY_NEWTONIAN, RHEOLOGY_BINGHAM = 0, 1
DYE_LEFT_RIGHT, DYE_TOP_BOTTOM, DYE_NONE = 0, 1, 2
WALL_PARTNER = 0xFFFFFFFF
WALL_IMPULSE_BINS = 32
IMPACT_BINS = 12
SE_BINS = 28


class _S(C.Structure):
    def to_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if isinstance(v, C.Structure):
                v = v.to_dict()
            elif isinstance(v, C.Array):
                v = list(v)
            out[name] = v
        return out

    def copy(self):
        c = type(self)()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(self))
        return c


class MillParams(_S):
    _fields_ = [("diameter_m", C.c_float), ("speed_mode", C.c_uint32), ("speed_value", C.c_float),
                ("direction", C.c_uint32)]


class MediaParams(_S):
    _fields_ = [(n, C.c_float) for n in (
        "ball_diameter_m", "fill_fraction", "packing_fraction_2d", "density_kg_m3",
        "restitution_ball_ball", "restitution_ball_wall", "friction_ball_ball", "friction_ball_wall",
        "friction_ball_ball_static", "friction_ball_wall_static", "friction_velocity_scale_m_s",
        "rolling_friction")]


class SlurryParams(_S):
    _fields_ = [("enabled", C.c_uint32), ("fill_fraction", C.c_float), ("density_kg_m3", C.c_float),
                ("viscosity_pa_s", C.c_float), ("rheology", C.c_uint32), ("yield_stress_pa", C.c_float),
                ("wall_no_slip", C.c_float), ("ball_no_slip", C.c_float), ("wettability", C.c_float),
                ("surface_tension_n_m", C.c_float), ("dye_pattern", C.c_uint32)]


class LiftersParams(_S):
    _fields_ = [("count", C.c_uint32), ("height_m", C.c_float), ("base_width_m", C.c_float),
                ("top_width_m", C.c_float), ("phase_deg", C.c_float)]


class SimulationParams(_S):
    _fields_ = [("resolution", C.c_uint32), ("substeps", C.c_uint32), ("pbf_iterations", C.c_uint32),
                ("dem_iterations", C.c_uint32), ("time_scale", C.c_float), ("frame_budget_ms", C.c_float),
                ("max_balls", C.c_uint32), ("reserved0", C.c_uint32), ("seed", C.c_uint64),
                ("coarse_graining_mode", C.c_uint32), ("coarse_graining_k", C.c_float)]


class Params(_S):
    _fields_ = [("mill", MillParams), ("media", MediaParams), ("slurry", SlurryParams),
                ("lifters", LiftersParams), ("simulation", SimulationParams)]


class Derived(_S):
    _fields_ = [("critical_speed_rpm", C.c_float), ("rpm", C.c_float), ("percent_critical", C.c_float),
                ("omega", C.c_float), ("radius_m", C.c_float), ("true_ball_count", C.c_float),
                ("eff_true_diameter_m", C.c_float), ("eff_diameter_m", C.c_float),
                ("eff_density_kg_m3", C.c_float), ("eff_ball_count", C.c_uint32),
                ("eff_scale_factor", C.c_float), ("effective_fluid_resolution", C.c_uint32),
                ("effective_substeps", C.c_uint32), ("fixed_sub_dt", C.c_float)]


class Drum(_S):
    _fields_ = [("radius_m", C.c_float), ("omega", C.c_float), ("lifters", LiftersParams)]


class FluidStepStats(_S):
    _fields_ = [("viscosity_iterations", C.c_uint32), ("mean_shear_rate_per_s", C.c_float),
                ("coupling_clamp_hits", C.c_uint32), ("wall_work_j", C.c_float),
                ("wall_impulse", C.c_float * 2), ("wall_angular_impulse", C.c_float),
                ("wall_normal_impulse_by_angle", C.c_float * WALL_IMPULSE_BINS),
                ("ke_delta_noslip_j", C.c_float), ("ke_delta_drag_j", C.c_float),
                ("ke_delta_buoyancy_j", C.c_float), ("ke_delta_viscosity_j", C.c_float),
                ("ke_delta_clamp_j", C.c_float)]


class DemStepStats(_S):
    _fields_ = [("wall_work_j", C.c_float), ("collision_count", C.c_uint32),
                ("impact_energy_histogram", C.c_uint32 * IMPACT_BINS), ("dissipated_energy_j", C.c_float),
                ("max_substep_displacement_over_diameter", C.c_float), ("coupling_work_j", C.c_float)]


class ImpactRecord(_S):
    _fields_ = [("kind", C.c_uint32), ("ball", C.c_uint32), ("partner", C.c_uint32),
                ("normal_speed", C.c_float), ("slip_speed", C.c_float), ("restitution", C.c_float)]


class StepCounters(_S):
    _fields_ = [(n, C.c_uint32) for n in (
        "density_iters", "cg_iters", "n_groups", "n_links", "links_in_range", "n_ball_pairs",
        "n_fluid_edges", "n_active_contacts", "n_coupling_items", "ccd_clamps")]


class BallMaterial(_S):
    _fields_ = [(n, C.c_float) for n in ("radius", "mass", "inertia", "true_radius")]


class FluidMaterial(_S):
    _fields_ = [(n, C.c_float) for n in ("particle_mass", "h", "rest_density")]


class EnergyBudget(_S):
    _fields_ = [(n, C.c_double) for n in (
        "elapsed_s", "shaft_work_j", "dem_wall_work_j", "fluid_wall_work_j", "ball_contact_dissipation_j",
        "fluid_wall_slip_j", "fluid_viscous_j", "fluid_clamp_removed_j", "interface_created_j",
        "delta_mechanical_j", "unattributed_j", "fluid_wall_angular_impulse")]


class Scalars(_S):
    _fields_ = [("drum_angle", C.c_float), ("power_draw_w", C.c_float), ("torque_nm", C.c_float),
                ("collision_rate_per_s", C.c_float), ("dissipated_power_w", C.c_float),
                ("max_substep_displacement_over_diameter", C.c_float), ("coupling_clamp_hits", C.c_uint32),
                ("viscosity_iterations", C.c_uint32), ("mean_shear_rate_per_s", C.c_float),
                ("reserved0", C.c_float), ("sim_time", C.c_double)]


class Options(_S):
    _fields_ = [("cg_fp64", C.c_uint32), ("block_threads", C.c_uint32), ("sweep_warps", C.c_uint32),
                ("spin_ns", C.c_uint32), ("mill_blocks", C.c_uint32), ("test_wait_limit_us", C.c_uint32),
                ("test_faults", C.c_uint32), ("block_regs", C.c_uint32), ("sweep_order", C.c_uint32)]


class ServerConfig(_S):
    _fields_ = [("memory_budget_bytes", C.c_uint64), ("max_active", C.c_uint32), ("block_threads", C.c_uint32),
                ("frame_dt", C.c_float), ("reserved", C.c_uint32 * 3)]


JOB_QUEUED, JOB_RUNNING, JOB_FINISHED, JOB_CANCELLED, JOB_FAILED = 0, 1, 2, 3, 4


class JobUpdate(_S):
    _fields_ = [("job_id", C.c_uint64), ("state", C.c_uint32), ("frames_done", C.c_uint32),
                ("frames_total", C.c_uint32), ("reserved0", C.c_uint32), ("scalars", Scalars),
                ("stress_histogram_rate", C.c_double * SE_BINS), ("state_hash", C.c_uint64),
                ("queued_s", C.c_double), ("first_frame_s", C.c_double)]


class ServerStats(_S):
    _fields_ = [("queued", C.c_uint32), ("active", C.c_uint32), ("finished_total", C.c_uint32),
                ("pending_updates", C.c_uint32), ("device_bytes_in_use", C.c_uint64), ("frames", C.c_uint64),
                ("last_frame_ms", C.c_float), ("last_kernel_ms", C.c_float)]


SURFACE_GRID = 128  # MG_SURFACE_GRID
SWEEP_MAX_SEEDS = 50  # MG_SWEEP_MAX_SEEDS
# most floats mg_fluid_surface can return: 1 + 9 * (2 segments in each of the (G - 1)^2 cells)
SURFACE_OUT_CAP = 1 + 9 * 2 * (SURFACE_GRID - 1) ** 2
METRIC_TOE_SHOULDER, METRIC_CENTROID, METRIC_POOL_EXTENT, METRIC_FREE_SURFACE = 0x01, 0x02, 0x04, 0x08
METRIC_POOL_DEPTH, METRIC_MIXING, METRIC_DENSITY = 0x10, 0x20, 0x40


class Metrics(_S):
    _fields_ = [("valid", C.c_uint32), ("toe_angle_rad", C.c_float), ("shoulder_angle_rad", C.c_float),
                ("charge_centroid_m", C.c_float * 2), ("pool_angle_min_rad", C.c_float),
                ("pool_angle_max_rad", C.c_float), ("free_surface_angle_rad", C.c_float),
                ("free_surface_offset_m", C.c_float), ("pool_depth_m", C.c_float), ("mixing_index", C.c_float),
                ("total_kinetic_energy_j", C.c_float), ("max_ball_overlap_fraction", C.c_float),
                ("max_ball_wall_overlap_fraction", C.c_float), ("max_fluid_density_error_fraction", C.c_float),
                ("mean_fluid_density_error_fraction", C.c_float),
                ("max_fluid_compression_error_fraction", C.c_float),
                ("mean_fluid_compression_error_fraction", C.c_float), ("drum_omega_rad_s", C.c_float),
                ("fluid_particle_count", C.c_uint32)]


class StressMetrics(_S):
    _fields_ = [("ball_mass_3d_kg", C.c_float), ("scale_energy_j", C.c_float),
                ("impacts_per_ball_per_s", C.c_float * 4), ("impacts_total_per_ball_per_s", C.c_float),
                ("mean_se_scaled", C.c_float * 4), ("mean_se_scaled_drop", C.c_float),
                ("mean_se_scaled_shear", C.c_float), ("stress_intensity_scaled", C.c_float),
                ("wall_power_per_ball_w", C.c_float), ("specific_power_w_per_kg", C.c_float),
                ("thresholds_scaled", C.c_float * 6), ("effective_power_per_ball_w", C.c_float * 6),
                ("reserved0", C.c_float), ("cumulative_wall_energy_per_ball_j", C.c_double),
                ("cumulative_specific_energy_j_per_kg", C.c_double),
                ("cumulative_effective_energy_per_ball_j", C.c_double * 6)]


SEED_VALUES = 23


class SeedResult(_S):
    _fields_ = [("seed", C.c_uint64), ("window_s", C.c_double), ("coarse_graining_factor", C.c_float),
                ("reserved0", C.c_float), ("values", C.c_double * SEED_VALUES),
                ("power_drift_rel_per_rev", C.c_double)]


P = C.POINTER
f32p = P(C.c_float)
u32p = P(C.c_uint32)
vp = C.c_void_p

# (name, restype, argtypes) of every entry point in include/millgpu.h
SIGNATURES = [
    ("sizeof_params", C.c_size_t, []),
    ("sizeof_fluid_stats", C.c_size_t, []),
    ("sizeof_dem_stats", C.c_size_t, []),
    ("params_default", C.c_int, [P(Params)]),
    ("params_validate", C.c_int, [P(Params), C.c_char_p, C.c_size_t]),
    ("preset_apply", C.c_int, [P(Params), C.c_char_p]),
    ("params_derived", C.c_int, [P(Params), P(Derived)]),
    ("sim_create", C.c_int, [P(Params), P(vp)]),
    ("sim_create_with_balls", C.c_int, [P(Params), f32p, C.c_uint32, P(vp)]),
    ("sim_destroy", None, [vp]),
    ("global_last_error", C.c_char_p, []),
    ("sim_step", C.c_int, [vp, C.c_float]),
    ("sim_step_fixed", C.c_int, [vp]),
    ("sim_reset_frame_stats", C.c_int, [vp]),
    ("sim_set_params", C.c_int, [vp, P(Params)]),
    ("sim_fixed_sub_dt", C.c_float, [vp]),
    ("sim_reset_energy_budget", C.c_int, [vp]),
    ("coupling_step_recorded", C.c_int, [vp, P(Drum), C.c_float, P(MediaParams), P(SlurryParams), C.c_uint32,
                                         C.c_uint32, C.c_float, P(FluidStepStats), P(DemStepStats),
                                         P(ImpactRecord), C.c_uint32, u32p]),
    ("fluid_step_coupled", C.c_int, [vp, P(Drum), C.c_float, P(SlurryParams), C.c_uint32, C.c_float,
                                     P(FluidStepStats), f32p, f32p, u32p, f32p]),
    ("dem_step_recorded", C.c_int, [vp, P(Drum), C.c_float, P(MediaParams), C.c_uint32, C.c_float, f32p, f32p,
                                    P(DemStepStats), P(ImpactRecord), C.c_uint32, u32p]),
    ("get_counts", C.c_int, [vp, u32p, u32p]),
    ("get_balls", C.c_int, [vp, f32p, f32p, f32p, f32p]),
    ("set_balls", C.c_int, [vp, C.c_uint32, f32p, f32p, f32p, f32p]),
    ("get_ball_material", C.c_int, [vp, P(BallMaterial)]),
    ("set_ball_material", C.c_int, [vp, P(BallMaterial)]),
    ("get_fluid", C.c_int, [vp, f32p, f32p, f32p, f32p, u32p]),
    ("set_fluid", C.c_int, [vp, C.c_uint32, f32p, f32p, f32p, f32p]),
    ("get_fluid_material", C.c_int, [vp, P(FluidMaterial)]),
    ("set_fluid_material", C.c_int, [vp, P(FluidMaterial)]),
    ("get_scalars", C.c_int, [vp, P(Scalars)]),
    ("energy_budget", C.c_int, [vp, P(EnergyBudget)]),
    ("state_hash", C.c_int, [vp, C.c_int, P(C.c_uint64)]),
    ("mixing_index", C.c_int, [vp, f32p, P(C.c_int)]),
    ("stress_histogram_rate", C.c_int, [vp, P(C.c_double)]),
    ("last_step_stats", C.c_int, [vp, P(FluidStepStats), P(DemStepStats), P(StepCounters)]),
    ("probe_grid", C.c_int, [f32p, C.c_uint32, C.c_float, P(C.c_int32), P(C.c_int64), u32p, C.c_uint32, u32p,
                             u32p, P(C.c_int)]),
    ("probe_candidate_pairs", C.c_int, [f32p, C.c_uint32, C.c_float, u32p, C.c_uint32, u32p]),
    ("probe_neighbor_lists", C.c_int, [f32p, C.c_uint32, C.c_float, u32p, u32p, C.c_uint32, u32p]),
    ("last_neighbor_lists", C.c_int, [vp, u32p, u32p, C.c_uint32, u32p]),
    ("last_ball_pairs", C.c_int, [vp, u32p, C.c_uint32, u32p]),
    ("stress_metrics", C.c_int, [vp, P(StressMetrics)]),
    ("metrics", C.c_int, [vp, P(Metrics)]),
    ("fluid_surface", C.c_int, [vp, f32p, C.c_uint32, u32p]),
    ("fluid_densities", C.c_int, [vp, f32p]),
    ("surface_field", C.c_int, [vp, f32p, f32p]),
    ("seed_value_name", C.c_char_p, [C.c_uint32]),
    ("seed_sweep", C.c_int, [P(Params), P(C.c_uint64), C.c_uint32, C.c_float, C.c_float, P(SeedResult)]),
    ("seed_combine", C.c_int, [P(SeedResult), C.c_uint32, P(C.c_double), P(C.c_double)]),
    ("seed_drift_per_rev", C.c_double, [P(C.c_double), C.c_uint32, C.c_double]),
]

# entry points only the device library exports
DEVICE_ONLY = [
    ("last_error", C.c_char_p, [vp]),
    ("sim_set_options", C.c_int, [vp, P(Options)]),
    ("sim_stream", C.c_int, [vp, P(vp)]),
    ("sim_last_kernel_ms", C.c_int, [vp, P(C.c_float), P(C.c_uint64)]),
    ("counter_totals", C.c_int, [vp, P(C.c_uint64), P(C.c_uint64), C.c_int]),
    ("stage_cycles", C.c_int, [vp, P(C.c_uint64), C.c_int]),
    ("batch_create", C.c_int, [P(Params), C.c_uint32, P(vp)]),
    ("batch_destroy", None, [vp]),
    ("batch_last_error", C.c_char_p, [vp]),
    ("batch_size", C.c_uint32, [vp]),
    ("batch_set_options", C.c_int, [vp, P(Options)]),
    ("batch_step_frames", C.c_int, [vp, C.c_uint32, C.c_float]),
    ("batch_scalars", C.c_int, [vp, P(Scalars)]),
    ("batch_mill", C.c_int, [vp, C.c_uint32, P(vp)]),
    ("batch_stream", C.c_int, [vp, P(vp)]),
    ("batch_last_kernel_ms", C.c_int, [vp, P(C.c_float), P(C.c_uint64)]),
    ("sim_footprint", C.c_int, [vp, P(C.c_uint64)]),
    ("server_create", C.c_int, [P(ServerConfig), P(vp)]),
    ("server_destroy", None, [vp]),
    ("server_last_error", C.c_char_p, [vp]),
    ("server_submit", C.c_int, [vp, P(Params), C.c_double, P(C.c_uint64)]),
    ("server_cancel", C.c_int, [vp, C.c_uint64]),
    ("server_submit_sweep", C.c_int, [vp, P(Params), C.c_uint32, C.c_float, C.c_float, P(C.c_uint64)]),
    ("server_sweep_result", C.c_int, [vp, C.c_uint64, P(SeedResult), P(C.c_double), P(C.c_double),
                                      P(C.c_uint32), P(C.c_uint32)]),
    ("server_sweep_release", C.c_int, [vp, C.c_uint64]),
    ("server_step", C.c_int, [vp]),
    ("server_poll", C.c_int, [vp, P(JobUpdate), C.c_uint32, u32p]),
    ("server_stats", C.c_int, [vp, P(ServerStats)]),
]

STAGE_NAMES = [
    "PBF predict + grid build", "density iterations", "ball overlap push (3.5)", "fluid cohesion (3.6a)",
    "ball adhesion (3.6b)", "wall projection (4-6)", "ball drag + buoyancy (6.5-6.6)", "density recompute",
    "viscosity: Morris weights (+ Bingham rates)", "viscosity: ball boundary pairs", "viscosity: squeeze links",
    "viscosity: CG solve (+ ball bookkeeping)", "mean_shear_rate", "fluid clamps/other (7.5-8)", "DEM step",
    "DEM: predict + broad phase + CCD", "DEM: projection sweeps", "DEM: friction", "DEM: restitution + rolling",
    "drag alone (6.5)", "DEM: projection predecessors", "DEM: projection levels", "DEM: level bucketing",
    "viscosity: CG setup (joint)", "drag: item lists", "drag: predecessors", "drag: sweep", "buoyancy: item lists",
    "buoyancy: predecessors", "buoyancy: sweep", "DEM: contact ordering", "viscosity: CG iterations (joint)",
    "drag sweep: ball prefetch (sum)", "drag sweep: ball waits (sum)", "drag sweep: ball chain work (sum)",
    "buoyancy sweep: ball prefetch (sum)", "buoyancy sweep: ball waits (sum)",
    "buoyancy sweep: ball chain work (sum)", "DEM: contact levels",
    "DEM: projection runs that failed their check"]
assert len(STAGE_NAMES) == 40


class Lib:
    """Binds the header's entry points of one shared library under `prefix`."""

    def __init__(self, path: str, prefix: str, extra=()):
        self.path = path
        self.prefix = prefix
        self.dll = C.CDLL(path)
        for name, res, args in list(SIGNATURES) + list(extra):
            fn = getattr(self.dll, prefix + name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)
