/*
 * millgpu.h -- C ABI of the B200 implementation of MillDynamics3's per-sub-step hot path
 * (PBF slurry + XPBD ball discs + two-way coupling), the drop-in for the Rust functions it names.
 *
 * Conventions (mirroring the reference's Rust API, crates/mill-core):
 *   - Every function returns an int status: MG_OK (0) on success, otherwise an MG_ERR_* code;
 *     mg_last_error(sim) / mg_global_last_error() give a message owned by the library.
 *   - Params are SI, field for field the reference's `Params` (params.rs:535-541) with the same
 *     names, units and defaults; enums are plain uint32 codes listed below.
 *   - State arrays are caller-owned, SoA, FP32, world coordinates with the drum centre at the
 *     origin (geometry.rs:112-114). Vec2 arrays are interleaved (x0, y0, x1, y1, ...).
 *   - The step is infallible in the reference (it sanitises NaN instead of failing); here a step
 *     fails only on device errors or on exceeding a buffer capacity, reported by status code.
 *   - Threading: one CUDA stream per handle; a handle is not thread-safe; distinct handles may be
 *     driven from distinct host threads.
 */
#ifndef MILLGPU_H
#define MILLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  MG_OK = 0,
  MG_ERR_INVALID_PARAMS = 1, /* Params::validate failed (params.rs:545-552) */
  MG_ERR_ARG = 2,            /* null pointer, size mismatch, unknown preset */
  MG_ERR_CUDA = 3,           /* a CUDA runtime call failed */
  MG_ERR_CAPACITY = 4,       /* a device buffer bound was exceeded (see mg_last_error) */
  MG_ERR_NO_DEVICE = 5,      /* no CUDA device / extension built without one */
  MG_ERR_STATE = 6           /* the handle is in an unusable state */
};

/* enum codes */
enum { MG_SPEED_RPM = 0, MG_SPEED_PERCENT_CRITICAL = 1 };
enum { MG_DIR_CCW = 0, MG_DIR_CW = 1 };
enum { MG_CG_AUTO = 0, MG_CG_OFF = 1, MG_CG_MANUAL = 2 };
enum { MG_RHEOLOGY_NEWTONIAN = 0, MG_RHEOLOGY_BINGHAM = 1 };
enum { MG_DYE_LEFT_RIGHT = 0, MG_DYE_TOP_BOTTOM = 1, MG_DYE_NONE = 2 };
enum { MG_IMPACT_BALL_BALL = 0, MG_IMPACT_BALL_WALL = 1 };
#define MG_WALL_PARTNER 0xFFFFFFFFu
#define MG_WALL_IMPULSE_BINS 32
#define MG_IMPACT_BINS 12
#define MG_SE_BINS 28

/* params.rs:53-60 MillParams */
typedef struct MgMillParams {
  float diameter_m;
  uint32_t speed_mode;
  float speed_value;
  uint32_t direction;
} MgMillParams;

/* params.rs:125-185 MediaParams */
typedef struct MgMediaParams {
  float ball_diameter_m, fill_fraction, packing_fraction_2d, density_kg_m3;
  float restitution_ball_ball, restitution_ball_wall, friction_ball_ball, friction_ball_wall;
  float friction_ball_ball_static, friction_ball_wall_static, friction_velocity_scale_m_s;
  float rolling_friction;
} MgMediaParams;

/* params.rs:297-345 SlurryParams */
typedef struct MgSlurryParams {
  uint32_t enabled;
  float fill_fraction, density_kg_m3, viscosity_pa_s;
  uint32_t rheology;
  float yield_stress_pa, wall_no_slip, ball_no_slip, wettability, surface_tension_n_m;
  uint32_t dye_pattern;
} MgSlurryParams;

/* params.rs:409-417 LiftersParams */
typedef struct MgLiftersParams {
  uint32_t count;
  float height_m, base_width_m, top_width_m, phase_deg;
} MgLiftersParams;

/* params.rs:452-491 SimulationParams */
typedef struct MgSimulationParams {
  uint32_t resolution, substeps, pbf_iterations, dem_iterations;
  float time_scale, frame_budget_ms;
  uint32_t max_balls, reserved0;
  uint64_t seed;
  uint32_t coarse_graining_mode;
  float coarse_graining_k;
} MgSimulationParams;

/* params.rs:535-541 Params */
typedef struct MgParams {
  MgMillParams mill;
  MgMediaParams media;
  MgSlurryParams slurry;
  MgLiftersParams lifters;
  MgSimulationParams simulation;
} MgParams;

/* Quantities derived from Params (params.rs:80-113, 558-726). */
typedef struct MgDerived {
  float critical_speed_rpm, rpm, percent_critical, omega, radius_m;
  float true_ball_count;
  float eff_true_diameter_m, eff_diameter_m, eff_density_kg_m3;
  uint32_t eff_ball_count;
  float eff_scale_factor;
  uint32_t effective_fluid_resolution, effective_substeps;
  float fixed_sub_dt;
} MgDerived;

/* geometry.rs:18-31 Drum */
typedef struct MgDrum {
  float radius_m, omega;
  MgLiftersParams lifters;
} MgDrum;

/* pbf.rs:874-917 FluidStepStats */
typedef struct MgFluidStepStats {
  uint32_t viscosity_iterations;
  float mean_shear_rate_per_s;
  uint32_t coupling_clamp_hits;
  float wall_work_j;
  float wall_impulse[2];
  float wall_angular_impulse;
  float wall_normal_impulse_by_angle[MG_WALL_IMPULSE_BINS];
  float ke_delta_noslip_j, ke_delta_drag_j, ke_delta_buoyancy_j, ke_delta_viscosity_j, ke_delta_clamp_j;
} MgFluidStepStats;

/* dem.rs:176-221 DemStepStats */
typedef struct MgDemStepStats {
  float wall_work_j;
  uint32_t collision_count;
  uint32_t impact_energy_histogram[MG_IMPACT_BINS];
  float dissipated_energy_j;
  float max_substep_displacement_over_diameter;
  float coupling_work_j;
} MgDemStepStats;

/* dem.rs:142-169 ImpactRecord (partner == MG_WALL_PARTNER for a wall impact) */
typedef struct MgImpactRecord {
  uint32_t kind, ball, partner;
  float normal_speed, slip_speed, restitution;
} MgImpactRecord;

/* Counters of the last sub-step (stage_timing.rs Counters semantics). */
typedef struct MgStepCounters {
  uint32_t density_iters, cg_iters, n_groups, n_links, links_in_range;
  uint32_t n_ball_pairs, n_fluid_edges, n_active_contacts;
  uint32_t n_coupling_items; /* entrained (ball, fluid) items of drag plus buoyancy */
  uint32_t ccd_clamps;       /* balls the wall CCD (dem.rs:674-706) held at their time of impact */
} MgStepCounters;

/* dem.rs:277-309 Balls' uniform material fields */
typedef struct MgBallMaterial {
  float radius, mass, inertia, true_radius;
} MgBallMaterial;

/* pbf.rs:1018-1028 FluidParticles' uniform material fields */
typedef struct MgFluidMaterial {
  float particle_mass, h, rest_density;
} MgFluidMaterial;

/* lib.rs:61-78 EnergyBudget */
typedef struct MgEnergyBudget {
  double elapsed_s, shaft_work_j, dem_wall_work_j, fluid_wall_work_j, ball_contact_dissipation_j;
  double fluid_wall_slip_j, fluid_viscous_j, fluid_clamp_removed_j, interface_created_j;
  double delta_mechanical_j, unattributed_j, fluid_wall_angular_impulse;
} MgEnergyBudget;

/* lib.rs:82-119 Simulation's scalar outputs */
typedef struct MgScalars {
  float drum_angle, power_draw_w, torque_nm, collision_rate_per_s, dissipated_power_w;
  float max_substep_displacement_over_diameter;
  uint32_t coupling_clamp_hits, viscosity_iterations;
  float mean_shear_rate_per_s, reserved0;
  double sim_time;
} MgScalars;

/* Device-path options. cg_fp64: 0 = the reference's sequential f32 inner products in the
 * viscosity solve, 1 = f64 inner products and residual norms. block_threads: threads per mill
 * block, a multiple of 32 up to 1024 (0 = 1024).
 * sweep_warps: warps that take balls in the per-ball drag and buoyancy sweeps (0 = default).
 * spin_ns: poll interval of a ball waiting for an earlier ball in those sweeps (0 = default).
 * mill_blocks: thread blocks that share a single mill's per-ball stages (adhesion, boundary
 * groups, squeeze links, drag and buoyancy item lists) in the handle's own launches: 0 = default
 * (16), 1 = the mill's block alone, at most 16 for handles from mg_sim_create /
 * mg_sim_create_with_balls; the mills of a batch or a server always run one block each (0 or 1).
 * None of them changes results.
 * test_wait_limit_us, test_faults: for tests of the failure path only (leave both 0).
 * test_wait_limit_us > 0 shortens the device's bounded waits (the mill block's wait for its helper
 * blocks, a ball's wait for earlier balls in the drag and buoyancy sweeps) from about a second or
 * more to about that many microseconds. test_faults bit 1: the mill's block waits for one more
 * helper block than was launched (a helper that never answers: its wait runs out, the step returns
 * MG_ERR_CUDA); bit 2: the drag sweep never flags ball 0 done (balls that share a fluid particle
 * with it wait until their limit runs out, the step returns MG_ERR_STATE).
 * block_regs: 0 = the register budget follows the block size (128 registers a thread up to 512
 * threads, 64 above); 64 = the 64-register build at any block size (two 512-thread blocks per
 * SM, for batches of small mills).
 * sweep_order: the order in which the warps of the drag and buoyancy sweeps take balls; 0 = by
 * dependency level (a ball after every ball it waits for, the chain's early links first), 1 =
 * ball index order. Results are the same either way. */
typedef struct MgOptions {
  uint32_t cg_fp64;
  uint32_t block_threads;
  uint32_t sweep_warps;
  uint32_t spin_ns;
  uint32_t mill_blocks;
  uint32_t test_wait_limit_us;
  uint32_t test_faults;
  uint32_t block_regs;
  uint32_t sweep_order;
} MgOptions;

typedef struct MgSim MgSim;

/* ---- sizes (layout checks for FFI bindings) ---- */
size_t mg_sizeof_params(void);
size_t mg_sizeof_fluid_stats(void);
size_t mg_sizeof_dem_stats(void);

/* ---- params.rs / presets.ts ---- */
/* Params::default() (params.rs:62-77,210-227,351-375,419-428,505-518) */
int mg_params_default(MgParams* out);
/* Params::validate() (params.rs:545-552); err receives the reference's message. */
int mg_params_validate(const MgParams* p, char* err, size_t err_len);
/* web/src/params/presets.ts:91-123 QUALITY_PRESETS by id ("realtime", "balanced", ...) */
int mg_preset_apply(MgParams* p, const char* id);
/* MillParams::{critical_speed_rpm,rpm,omega}, Params::{true_ball_count, effective_media,
 * effective_fluid_resolution, effective_substeps}, Simulation::fixed_sub_dt */
int mg_params_derived(const MgParams* p, MgDerived* out);

/* ---- lib.rs Simulation ---- */
/* Simulation::new (lib.rs:126-128) */
int mg_sim_create(const MgParams* p, MgSim** out);
/* Simulation::with_initial_balls (lib.rs:134-136); xy holds n interleaved positions */
int mg_sim_create_with_balls(const MgParams* p, const float* xy, uint32_t n, MgSim** out);
void mg_sim_destroy(MgSim* sim);
const char* mg_last_error(const MgSim* sim);
const char* mg_global_last_error(void);
int mg_sim_set_options(MgSim* sim, const MgOptions* opt);
/* Simulation::step (lib.rs:456-464): effective_substeps() sub-steps of dt/n each */
int mg_sim_step(MgSim* sim, float dt);
/* Simulation::step_fixed (lib.rs:438-441) */
int mg_sim_step_fixed(MgSim* sim);
/* Simulation::reset_frame_stats (lib.rs:449-452) */
int mg_sim_reset_frame_stats(MgSim* sim);
/* Simulation::set_params (lib.rs:270-274) */
int mg_sim_set_params(MgSim* sim, const MgParams* p);
/* Simulation::fixed_sub_dt (lib.rs:426-428) */
float mg_sim_fixed_sub_dt(const MgSim* sim);
/* Simulation::reset_energy_budget (lib.rs:211-214) */
int mg_sim_reset_energy_budget(MgSim* sim);

/* ---- the path itself: coupling.rs:71-96 step_recorded ----
 * Runs one coupled sub-step (fluid first, then the balls with the fluid's impulses) on the
 * handle's state, in place. Impact records are written to `out` (up to `cap`); *n_out receives
 * the full count (a count above cap means records were dropped). Any stats pointer may be NULL. */
int mg_coupling_step_recorded(MgSim* sim, const MgDrum* drum, float drum_angle, const MgMediaParams* media,
                              const MgSlurryParams* slurry, uint32_t dem_iterations, uint32_t pbf_iterations,
                              float dt, MgFluidStepStats* fluid_stats, MgDemStepStats* dem_stats,
                              MgImpactRecord* out, uint32_t cap, uint32_t* n_out);
/* FluidParticles::step_coupled (pbf.rs:1174-2365): the fluid half alone; impulses (2*n_balls),
 * angular (n_balls), clamp_hits and fluid_momentum (2) receive CouplingImpulses (coupling.rs:37-63). */
int mg_fluid_step_coupled(MgSim* sim, const MgDrum* drum, float drum_angle, const MgSlurryParams* slurry,
                          uint32_t iterations, float dt, MgFluidStepStats* stats, float* impulses, float* angular,
                          uint32_t* clamp_hits, float* fluid_momentum);
/* DemState::step_recorded (dem.rs:530-1066): the ball half alone; impulses/angular may be NULL
 * (no external impulses, DemState::step). */
int mg_dem_step_recorded(MgSim* sim, const MgDrum* drum, float drum_angle, const MgMediaParams* media,
                         uint32_t iterations, float dt, const float* impulses, const float* angular,
                         MgDemStepStats* stats, MgImpactRecord* out, uint32_t cap, uint32_t* n_out);

/* ---- state I/O ---- */
int mg_get_counts(const MgSim* sim, uint32_t* n_balls, uint32_t* n_fluid);
int mg_get_balls(MgSim* sim, float* x, float* v, float* theta, float* omega);
int mg_set_balls(MgSim* sim, uint32_t n, const float* x, const float* v, const float* theta, const float* omega);
int mg_get_ball_material(const MgSim* sim, MgBallMaterial* out);
int mg_set_ball_material(MgSim* sim, const MgBallMaterial* m);
/* guess may be NULL; *guess_len receives the viscous warm-start length (0 or n_fluid). */
int mg_get_fluid(MgSim* sim, float* x, float* v, float* dye, float* guess, uint32_t* guess_len);
/* guess may be NULL (empty warm start, as after FluidParticles::seed_lattice). */
int mg_set_fluid(MgSim* sim, uint32_t n, const float* x, const float* v, const float* dye, const float* guess);
int mg_get_fluid_material(const MgSim* sim, MgFluidMaterial* out);
int mg_set_fluid_material(MgSim* sim, const MgFluidMaterial* m);

/* ---- outputs ---- */
int mg_get_scalars(MgSim* sim, MgScalars* out);
/* Simulation::energy_budget (lib.rs:218-229) */
int mg_energy_budget(MgSim* sim, MgEnergyBudget* out);
/* FNV-1a over the f32 bits of the state (examples/perf_probe.rs:230-262) */
int mg_state_hash(MgSim* sim, int extended, uint64_t* out);
/* metrics::mixing_index (metrics.rs:506-576); *valid = 0 for None */
int mg_mixing_index(MgSim* sim, float* out, int* valid);

/* metrics::Metrics, the fields metrics::compute fills (metrics.rs:78-273): charge toe/shoulder,
 * centroid, slurry pool extent and depth, free-surface line, mixing index, ball kinetic energy,
 * ball-ball and ball-wall overlap, fluid density and compression errors. Option fields are
 * present when their bit is set in `valid`. */
#define MG_METRIC_TOE_SHOULDER 0x01u
#define MG_METRIC_CENTROID 0x02u
#define MG_METRIC_POOL_EXTENT 0x04u
#define MG_METRIC_FREE_SURFACE 0x08u
#define MG_METRIC_POOL_DEPTH 0x10u
#define MG_METRIC_MIXING 0x20u
#define MG_METRIC_DENSITY 0x40u /* the four fluid density / compression error fields */
typedef struct MgMetrics {
  uint32_t valid;
  float toe_angle_rad, shoulder_angle_rad;
  float charge_centroid_m[2];
  float pool_angle_min_rad, pool_angle_max_rad;
  float free_surface_angle_rad, free_surface_offset_m;
  float pool_depth_m;
  float mixing_index;
  float total_kinetic_energy_j;
  float max_ball_overlap_fraction, max_ball_wall_overlap_fraction;
  float max_fluid_density_error_fraction, mean_fluid_density_error_fraction;
  float max_fluid_compression_error_fraction, mean_fluid_compression_error_fraction;
  float drum_omega_rad_s;
  uint32_t fluid_particle_count;
} MgMetrics;
/* metrics::compute(balls, fluid, drum, drum_angle) (metrics.rs:195-273) on the handle's current
 * state, as one kernel launch on the handle's stream. The launch rebuilds the fluid neighbour
 * lists for the current positions in the handle's sub-step scratch, so mg_last_neighbor_lists
 * afterwards returns those. */
int mg_metrics(MgSim* sim, MgMetrics* out);

/* Free-surface extraction for rendering. */
#define MG_SURFACE_GRID 128 /* grid points per axis over [-R, R] (surface.rs:27) */
/* Simulation::fluid_surface (lib.rs:354-361: surface::extract_surface, surface.rs:233-272) on the
 * handle's current state, flattened as mill-wasm's fluid_surface returns it (flatten_polygons,
 * surface.rs:420-430): [n_polys, len_0, x, y, ..., len_1, x, y, ...], world frame. Two kernel
 * launches on the handle's stream (splatted field; contour, chaining, smoothing and wall
 * projection). *len receives the number of floats (1 when there is no surface). out may be NULL
 * to query the length; MG_ERR_CAPACITY when out is non-NULL and cap < *len (nothing copied). */
int mg_fluid_surface(MgSim* sim, float* out, uint32_t cap, uint32_t* len);
/* The masked occupancy field build_field returns (surface.rs:84-131), MG_SURFACE_GRID^2 floats,
 * row gj * MG_SURFACE_GRID + gi, and analytic_phi_full (surface.rs:71-74) of the fluid. No
 * counterpart in the reference's public API: build_field is private there; this exposes it for
 * checks against the oracle. */
int mg_surface_field(MgSim* sim, float* field, float* phi_full);
/* FluidParticles::densities (pbf.rs:1124-1145) of the current positions: out receives n_fluid
 * floats. Computed by the mg_metrics launch (which it runs). */
int mg_fluid_densities(MgSim* sim, float* out);
/* StressAccum::histogram_rate (stress.rs:174-176), 28 bins per second */
int mg_stress_histogram_rate(MgSim* sim, double* out28);
/* stats of the last sub-step taken by any step call */
int mg_last_step_stats(MgSim* sim, MgFluidStepStats* fluid, MgDemStepStats* dem, MgStepCounters* ctr);

/* ---- measurement ----
 * The CUDA stream the handle launches on (a cudaStream_t), for event timing by the caller. */
int mg_sim_stream(MgSim* sim, void** stream);
/* Device duration (CUDA events) of the last kernel launch, and the number of launches so far. */
int mg_sim_last_kernel_ms(MgSim* sim, float* ms, uint64_t* launches);
/* Sums of every MgStepCounters field over all sub-steps since creation (or the last reset),
 * in field order, and the number of sub-steps summed. */
int mg_counter_totals(MgSim* sim, uint64_t* totals10, uint64_t* n_substeps, int reset);
/* Device cycles per stage summed over all sub-steps since creation (or the last reset): slots
 * 0-14 are the reference's stage_timing.rs stages (predict + grid, density, push, cohesion,
 * adhesion, wall 4-6, drag + buoyancy, density recompute, Morris weights, ball boundary pairs,
 * squeeze links, CG, mean shear rate, clamps, DEM), 15-18 split the DEM step (predict + broad
 * phase, projection, friction, restitution + rolling), 19 is drag alone and 20-31 split the
 * sweeps further (DEM predecessors, levels, level bucketing, contact ordering; drag and
 * buoyancy item lists, predecessors and sweeps; 23 and 31 the joint viscosity solve's setup and
 * iterations, 11 then keeping its bookkeeping). 32-37 are not wall-clock slots: they sum over
 * balls the cycles the drag (32-34) and buoyancy (35-37) sweeps spent prefetching each ball,
 * waiting for earlier balls and running the ball's dependent part; 38 the dependency levels of
 * the active contacts (friction and restitution); 39 the projection runs whose check that the
 * pairs left out stayed apart failed (the run that follows adds to 20-22 and 16). 40 slots in
 * all. */
int mg_stage_cycles(MgSim* sim, uint64_t* cycles40, int reset);

/* ---- parity probes of the grid stage (grid.rs, pbf.rs:262-288) ----
 * Run the device grid build / candidate-pair / neighbour-list code on caller points. */
int mg_probe_grid(const float* xy, uint32_t n, float cell, int32_t* min_cxy, int64_t* wh, uint32_t* cell_start,
                  uint32_t cell_cap, uint32_t* indices, uint32_t* n_cells_out, int* dense_out);
int mg_probe_candidate_pairs(const float* xy, uint32_t n, float cell, uint32_t* pairs, uint32_t cap, uint32_t* n_out);
int mg_probe_neighbor_lists(const float* xy, uint32_t n, float h, uint32_t* offsets, uint32_t* nbrs, uint32_t cap,
                            uint32_t* n_edges);
/* The neighbour CSR of mg_probe_neighbor_lists without allocating anything. No reference
 * counterpart: it exists for callers that cannot allocate device memory per call (a loop held to
 * a fixed memory budget, or one that must not synchronise the device). All pointers are DEVICE
 * pointers the caller owns: xy_dev (2n floats), offsets_dev (n + 1), nbrs_dev (cap),
 * n_edges_dev (1; the full edge count, also when it exceeds cap) and status_dev (1; 0 or error
 * bits: 1 = cap too small, nothing written to nbrs_dev; 4 = a cell key saturated). Runs
 * asynchronously on `stream` (a cudaStream_t; NULL = the legacy default stream); the grid scratch
 * is one fixed static device array (at most 16384 points per call; a larger n returns
 * MG_ERR_CAPACITY). Calls on one device share that scratch and must not overlap (issue them on
 * one stream). The first call on a device resolves the scratch address; make it before capturing
 * a stream. The address is kept for the life of the process and belongs to the device's primary
 * context (the CUDA runtime's): do not call cudaDeviceReset between calls, and do not call it with
 * another context current on the device. */
int mg_neighbor_lists_noalloc(const float* xy_dev, uint32_t n, float h, uint32_t* offsets_dev, uint32_t* nbrs_dev,
                              uint32_t cap, uint32_t* n_edges_dev, uint32_t* status_dev, void* stream);
/* neighbour CSR / ball pair list of the last fluid / ball sub-step taken on this handle */
int mg_last_neighbor_lists(MgSim* sim, uint32_t* offsets, uint32_t* nbrs, uint32_t cap, uint32_t* n_edges);
int mg_last_ball_pairs(MgSim* sim, uint32_t* pairs, uint32_t cap, uint32_t* n_out);

/* ---- batches: many independent mills per launch (batch::run_seed's unit of work, batch.rs:40-191,
 * run many at a time). No single reference counterpart: the reference steps one Simulation at a
 * time. Each mill is an ordinary Simulation (params[i], its own seed) whose sub-steps run as one
 * thread block of a shared launch; a mill's results are identical alone or in a batch. */
typedef struct MgBatch MgBatch;
int mg_batch_create(const MgParams* params, uint32_t n_mills, MgBatch** out);
void mg_batch_destroy(MgBatch* batch);
const char* mg_batch_last_error(const MgBatch* batch);
uint32_t mg_batch_size(const MgBatch* batch);
int mg_batch_set_options(MgBatch* batch, const MgOptions* opt);
/* Simulation::step(frame_dt) on every mill, `frames` times (each mill its own effective_substeps). */
int mg_batch_step_frames(MgBatch* batch, uint32_t frames, float frame_dt);
/* Simulation scalars of every mill (n_mills entries). */
int mg_batch_scalars(MgBatch* batch, MgScalars* out);
/* Borrows mill i's handle for the per-mill accessors (mg_get_balls, mg_energy_budget,
 * mg_stress_histogram_rate, mg_state_hash ...). Owned by the batch: do not destroy it. */
int mg_batch_mill(MgBatch* batch, uint32_t i, MgSim** out);
int mg_batch_stream(MgBatch* batch, void** stream);
/* Device duration of the last frame launch and the number of frame launches so far. */
int mg_batch_last_kernel_ms(MgBatch* batch, float* ms, uint64_t* launches);
/* Device memory a handle holds (its arena plus launch blocks), for admission by footprint. */
int mg_sim_footprint(const MgSim* sim, uint64_t* device_bytes);

/* ---- grinding-proxy statistics and seed sweeps ----
 * StressMetrics (stress.rs:186-273), what Simulation::metrics().stress reports (lib.rs:370-390):
 * per-ball impact rates by class (ball-ball drop, ball-ball shear, ball-wall drop, ball-wall
 * shear), mean scaled stress energies, wall power per ball, effective power above the six
 * thresholds (multiples of m g d) and the cumulative energies. */
typedef struct MgStressMetrics {
  float ball_mass_3d_kg, scale_energy_j;
  float impacts_per_ball_per_s[4];
  float impacts_total_per_ball_per_s;
  float mean_se_scaled[4];
  float mean_se_scaled_drop, mean_se_scaled_shear, stress_intensity_scaled;
  float wall_power_per_ball_w, specific_power_w_per_kg;
  float thresholds_scaled[6];
  float effective_power_per_ball_w[6];
  float reserved0;
  double cumulative_wall_energy_per_ball_j, cumulative_specific_energy_j_per_kg;
  double cumulative_effective_energy_per_ball_j[6];
} MgStressMetrics;
int mg_stress_metrics(MgSim* sim, MgStressMetrics* out);

/* batch::run_seed (batch.rs:40-107): window means of one seed's run. values[k] is named by
 * mg_seed_value_name(k): the 16 per-frame stress scalars averaged over the measured frames, then
 * the exact window powers from the cumulative energies (specific power and the six effective
 * powers per ball). */
#define MG_SEED_VALUES 23
typedef struct MgSeedResult {
  uint64_t seed;
  double window_s;                /* simulated seconds averaged over */
  float coarse_graining_factor;   /* k of the run; the statistics are meaningless for k > 1 */
  float reserved0;
  double values[MG_SEED_VALUES];
  double power_drift_rel_per_rev; /* least-squares slope of the wall power per revolution / mean */
} MgSeedResult;
const char* mg_seed_value_name(uint32_t k);
/* run_seed for every seeds[i] (replacing params->simulation.seed): warm-up revolutions, then
 * measured revolutions (>= 1). The device library advances all seeds together, one launch per
 * frame (a batch); each seed's numbers are those of run_seed on that seed alone. */
int mg_seed_sweep(const MgParams* params, const uint64_t* seeds, uint32_t n_seeds, float warmup_revolutions,
                  float measure_revolutions, MgSeedResult* out);
/* batch::combine (batch.rs:161-190): per value, the mean over seeds and its standard error
 * (sample standard deviation with n - 1, over sqrt(n); 0 for one seed). */
int mg_seed_combine(const MgSeedResult* results, uint32_t n, double* mean, double* std_err);
/* batch.rs:141-159 drift_per_rev: slope of y against the frame index relative to the mean of y,
 * per revolution of frames_per_rev frames (0 for fewer than two samples or a zero mean). */
double mg_seed_drift_per_rev(const double* y, uint32_t n, double frames_per_rev);

/* ---- request server: continuous batching of mill jobs. No single reference counterpart (the
 * reference runs one Simulation per web worker, worker.ts:138-142, and seed sweeps one after
 * another, batch.rs:40-191). Jobs (Params + a simulated horizon) wait in a queue and are admitted
 * oldest first whenever the device bytes of their state fit under the budget; each
 * mg_server_step advances every admitted job by one frame in one launch and retires the jobs
 * that reached their horizon. A job's results are identical to the same mill stepped alone. */
typedef struct MgServer MgServer;
typedef struct MgServerConfig {
  uint64_t memory_budget_bytes; /* device bytes all admitted jobs may hold together (0 = 150 GiB) */
  uint32_t max_active;          /* jobs advanced per step at most (0 = 1024) */
  uint32_t block_threads;       /* 0 = default */
  float frame_dt;               /* simulated seconds per frame (0 = 1/60) */
  uint32_t reserved[3];
} MgServerConfig;
enum { MG_JOB_QUEUED = 0, MG_JOB_RUNNING = 1, MG_JOB_FINISHED = 2, MG_JOB_CANCELLED = 3, MG_JOB_FAILED = 4 };
/* One job's state after a frame (RUNNING) or at its end (FINISHED / CANCELLED / FAILED). */
typedef struct MgJobUpdate {
  uint64_t job_id;
  uint32_t state, frames_done, frames_total, reserved0;
  MgScalars scalars;                          /* power, torque, ... after the job's latest frame */
  double stress_histogram_rate[MG_SE_BINS];   /* StressAccum::histogram_rate (stress.rs:174-238) */
  uint64_t state_hash;                        /* extended state hash when FINISHED, else 0 */
  double queued_s;                            /* wall seconds from submission to admission */
  double first_frame_s;                       /* wall seconds from submission to its first frame's end */
} MgJobUpdate;
typedef struct MgServerStats {
  uint32_t queued, active, finished_total, pending_updates;
  uint64_t device_bytes_in_use, frames;
  float last_frame_ms, last_kernel_ms;        /* wall time of the last step; device time of its launch */
} MgServerStats;
int mg_server_create(const MgServerConfig* cfg, MgServer** out);
void mg_server_destroy(MgServer* server);
const char* mg_server_last_error(const MgServer* server);
/* Queues a job of ceil(horizon_s / frame_dt) frames; *job_id identifies it in the updates. */
int mg_server_submit(MgServer* server, const MgParams* p, double horizon_s, uint64_t* job_id);
/* A queued job leaves at once, a running one before the next frame (a CANCELLED update). */
int mg_server_cancel(MgServer* server, uint64_t job_id);
/* Admits what fits, advances every running job by one frame, retires the finished ones. */
int mg_server_step(MgServer* server);
/* Hands out (and forgets) up to cap pending updates, oldest first; *n_out receives the count. */
int mg_server_poll(MgServer* server, MgJobUpdate* out, uint32_t cap, uint32_t* n_out);
int mg_server_stats(MgServer* server, MgServerStats* out);

/* Seed-sweep jobs: the web batch planner's repeat runs (web/src/batch/plan.ts, protocol.ts) as a
 * job type of the serving loop. A sweep queues one job per seed 1..=n_seeds (the literal numbers,
 * plan.ts:29-32) of the same Params; each runs batch::run_seed's window (warm-up revolutions,
 * then measured revolutions, batch.rs:40-107) while other jobs share the launches, and streams
 * ordinary job updates. The planner's rules are enforced at submission: 1 <= n_seeds <=
 * MG_SWEEP_MAX_SEEDS, warm-up >= 0, measured revolutions an integer >= 1, a drum speed > 0, and
 * no coarse-graining (k = 1; plan.ts:13-26, 78-91). mg_server_cancel(sweep_id) cancels every seed. */
#define MG_SWEEP_MAX_SEEDS 50
int mg_server_submit_sweep(MgServer* server, const MgParams* p, uint32_t n_seeds, float warmup_revolutions,
                           float measure_revolutions, uint64_t* sweep_id);
/* *state: MG_JOB_QUEUED / RUNNING until every seed has finished, then FINISHED (or CANCELLED /
 * FAILED if a seed was); *seeds_finished counts finished seeds. Once FINISHED, results[n_seeds]
 * receives each seed's MgSeedResult (seed order) and mean / std_err[MG_SEED_VALUES] their
 * batch::combine (any of the three may be NULL). */
int mg_server_sweep_result(MgServer* server, uint64_t sweep_id, MgSeedResult* results, double* mean,
                           double* std_err, uint32_t* state, uint32_t* seeds_finished);
/* Forgets a sweep's record (read its result first): seeds still queued or running are cancelled,
 * and the id is unknown afterwards. When one seed fails, the sweep is FAILED and its other seeds
 * leave without this call (queued ones at the next admission, running ones before the next
 * frame). */
int mg_server_sweep_release(MgServer* server, uint64_t sweep_id);

#ifdef __cplusplus
}
#endif

#endif /* MILLGPU_H */
