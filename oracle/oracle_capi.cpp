// Oracle C API (test infrastructure only): the same entry points as include/millgpu.h with an
// `or_` prefix, over the CPU restatement, so tests drive the oracle and the device library
// through identical calls. Uses the public header for POD layouts only.
#include <algorithm>
#include <cstring>
#include <string>

#include "../include/millgpu.h"
#include "oracle_core.hpp"

using namespace orc;

static_assert(sizeof(MgParams) == sizeof(Params), "param layout");
static_assert(sizeof(MgMediaParams) == sizeof(MediaParams), "media layout");
static_assert(sizeof(MgSlurryParams) == sizeof(SlurryParams), "slurry layout");
static_assert(sizeof(Real) != sizeof(float) || sizeof(MgFluidStepStats) == sizeof(FluidStepStats),
              "fluid stats layout");
static_assert(sizeof(Real) != sizeof(float) || sizeof(MgDemStepStats) == sizeof(DemStepStats), "dem stats layout");
static_assert(sizeof(MgImpactRecord) == sizeof(ImpactRecord), "impact layout");
static_assert(sizeof(MgStepCounters) == sizeof(StepCounters), "counter layout");

// The stats structs hold Real (f32 in the parity oracle, where this is a plain copy; f64 in the
// FP64 oracle, rounded to the ABI's f32 here).
static void to_mg(const FluidStepStats& a, MgFluidStepStats* o) {
  o->viscosity_iterations = a.viscosity_iterations;
  o->mean_shear_rate_per_s = (float)a.mean_shear_rate_per_s;
  o->coupling_clamp_hits = a.coupling_clamp_hits;
  o->wall_work_j = (float)a.wall_work_j;
  o->wall_impulse[0] = (float)a.wall_impulse[0];
  o->wall_impulse[1] = (float)a.wall_impulse[1];
  o->wall_angular_impulse = (float)a.wall_angular_impulse;
  for (int k = 0; k < WALL_IMPULSE_BINS; ++k) o->wall_normal_impulse_by_angle[k] = (float)a.wall_normal_impulse_by_angle[k];
  o->ke_delta_noslip_j = (float)a.ke_delta_noslip_j;
  o->ke_delta_drag_j = (float)a.ke_delta_drag_j;
  o->ke_delta_buoyancy_j = (float)a.ke_delta_buoyancy_j;
  o->ke_delta_viscosity_j = (float)a.ke_delta_viscosity_j;
  o->ke_delta_clamp_j = (float)a.ke_delta_clamp_j;
}
static void to_mg(const DemStepStats& a, MgDemStepStats* o) {
  o->wall_work_j = (float)a.wall_work_j;
  o->collision_count = a.collision_count;
  for (int k = 0; k < IMPACT_BINS; ++k) o->impact_energy_histogram[k] = a.impact_energy_histogram[k];
  o->dissipated_energy_j = (float)a.dissipated_energy_j;
  o->max_substep_displacement_over_diameter = (float)a.max_substep_displacement_over_diameter;
  o->coupling_work_j = (float)a.coupling_work_j;
}
static std::vector<Real> reals(const float* a, uint32_t n) { return std::vector<Real>(a, a + n); }
template <class V> static void put_reals(const V& v, float* out) {
  if (out) for (size_t k = 0; k < v.size(); ++k) out[k] = (float)v[k];
}

struct OrSim {
  Simulation sim;
  std::string err;
};

static thread_local std::string g_err;

static Params to_p(const MgParams* p) { Params q; std::memcpy(&q, p, sizeof(q)); return q; }
static Drum to_drum(const MgDrum* d) {
  Drum q;
  q.radius_m = d->radius_m;
  q.omega = d->omega;
  std::memcpy(&q.lifters, &d->lifters, sizeof(q.lifters));
  return q;
}
static std::vector<Vec2> vecs(const float* xy, uint32_t n) {
  std::vector<Vec2> v(n);
  for (uint32_t i = 0; i < n; ++i) v[i] = Vec2(xy[2 * i], xy[2 * i + 1]);
  return v;
}
static void put(const std::vector<Vec2>& v, float* out) {
  if (!out) return;
  for (size_t i = 0; i < v.size(); ++i) { out[2 * i] = v[i].x; out[2 * i + 1] = v[i].y; }
}

extern "C" {

size_t or_sizeof_params(void) { return sizeof(MgParams); }
size_t or_sizeof_fluid_stats(void) { return sizeof(MgFluidStepStats); }
size_t or_sizeof_dem_stats(void) { return sizeof(MgDemStepStats); }

int or_params_default(MgParams* out) {
  Params p = params_default();
  std::memcpy(out, &p, sizeof(p));
  return MG_OK;
}
int or_params_validate(const MgParams* p, char* err, size_t n) {
  std::string e;
  if (params_validate(to_p(p), &e)) return MG_OK;
  if (err && n) { std::strncpy(err, e.c_str(), n - 1); err[n - 1] = 0; }
  return MG_ERR_INVALID_PARAMS;
}
int or_preset_apply(MgParams* p, const char* id) {
  Params q = to_p(p);
  if (!preset_apply(&q, id)) return MG_ERR_ARG;
  std::memcpy(p, &q, sizeof(q));
  return MG_OK;
}
int or_params_derived(const MgParams* pp, MgDerived* o) {
  Params p = to_p(pp);
  EffectiveMedia e = effective_media(p);
  o->critical_speed_rpm = critical_speed_rpm(p.mill);
  o->rpm = mill_rpm(p.mill);
  o->percent_critical = mill_percent_critical(p.mill);
  o->omega = mill_omega(p.mill);
  o->radius_m = mill_radius(p.mill);
  o->true_ball_count = true_ball_count(p);
  o->eff_true_diameter_m = e.true_diameter_m;
  o->eff_diameter_m = e.diameter_m;
  o->eff_density_kg_m3 = e.density_kg_m3;
  o->eff_ball_count = e.ball_count;
  o->eff_scale_factor = e.scale_factor;
  o->effective_fluid_resolution = effective_fluid_resolution(p);
  o->effective_substeps = effective_substeps(p);
  o->fixed_sub_dt = 1.0f / (60.0f * (float)std::max(effective_substeps(p), 1u));
  return MG_OK;
}

static int create(const MgParams* p, const float* xy, uint32_t n, OrSim** out) {
  OrSim* s = new OrSim();
  std::vector<Vec2> init;
  if (xy) init = vecs(xy, n);
  std::string e;
  if (!Simulation::build(to_p(p), xy ? &init : nullptr, &s->sim, &e)) {
    g_err = e;
    delete s;
    return MG_ERR_INVALID_PARAMS;
  }
  *out = s;
  return MG_OK;
}
int or_sim_create(const MgParams* p, OrSim** out) { return create(p, nullptr, 0, out); }
int or_sim_create_with_balls(const MgParams* p, const float* xy, uint32_t n, OrSim** out) {
  return create(p, xy, n, out);
}
void or_sim_destroy(OrSim* s) { delete s; }
const char* or_global_last_error(void) { return g_err.c_str(); }
int or_sim_set_cg_fp64(OrSim* s, int on) { s->sim.opt.cg_fp64 = on; return MG_OK; }
int or_sim_step(OrSim* s, float dt) { s->sim.step(dt); return MG_OK; }
int or_sim_step_fixed(OrSim* s) { s->sim.step_fixed(); return MG_OK; }
int or_sim_reset_frame_stats(OrSim* s) { s->sim.reset_frame_stats(); return MG_OK; }
int or_sim_set_params(OrSim* s, const MgParams* p) {
  std::string e;
  if (!params_validate(to_p(p), &e)) { s->err = e; return MG_ERR_INVALID_PARAMS; }
  s->sim.params = to_p(p);
  return MG_OK;
}
float or_sim_fixed_sub_dt(const OrSim* s) { return s->sim.fixed_sub_dt(); }
int or_sim_reset_energy_budget(OrSim* s) {
  s->sim.energy_budget = EnergyBudget();
  s->sim.energy_budget_e0 = s->sim.total_mechanical_energy_j();
  return MG_OK;
}

int or_coupling_step_recorded(OrSim* s, const MgDrum* drum, float drum_angle, const MgMediaParams* media,
                              const MgSlurryParams* slurry, uint32_t dem_it, uint32_t pbf_it, float dt,
                              MgFluidStepStats* fstats, MgDemStepStats* dstats, MgImpactRecord* out, uint32_t cap,
                              uint32_t* n_out) {
  Drum d = to_drum(drum);
  MediaParams m;
  std::memcpy(&m, media, sizeof(m));
  SlurryParams sl;
  std::memcpy(&sl, slurry, sizeof(sl));
  CouplingImpulses imp;
  FluidStepStats fs;
  StepCounters ctr;
  fluid_step_coupled(&s->sim.fluid, d, drum_angle, sl, pbf_it, dt, s->sim.balls, &imp, &fs, &ctr, &s->sim.dbg,
                     s->sim.opt);
  std::vector<ImpactRecord> recs;
  DemStepStats ds = dem_step_recorded(&s->sim.balls, d, drum_angle, m, dem_it, dt, &imp, &recs, &ctr, &s->sim.dbg);
  s->sim.last_counters = ctr;
  s->sim.fluid_stats = fs;
  s->sim.last_dem_stats = ds;
  if (fstats) to_mg(fs, fstats);
  if (dstats) to_mg(ds, dstats);
  if (n_out) *n_out = (uint32_t)recs.size();
  if (out)
    for (size_t k = 0; k < recs.size() && k < cap; ++k) std::memcpy(&out[k], &recs[k], sizeof(ImpactRecord));
  return MG_OK;
}

int or_fluid_step_coupled(OrSim* s, const MgDrum* drum, float drum_angle, const MgSlurryParams* slurry,
                          uint32_t it, float dt, MgFluidStepStats* fstats, float* impulses, float* angular,
                          uint32_t* clamp_hits, float* fluid_momentum) {
  Drum d = to_drum(drum);
  SlurryParams sl;
  std::memcpy(&sl, slurry, sizeof(sl));
  CouplingImpulses imp;
  FluidStepStats fs;
  StepCounters ctr;
  fluid_step_coupled(&s->sim.fluid, d, drum_angle, sl, it, dt, s->sim.balls, &imp, &fs, &ctr, &s->sim.dbg,
                     s->sim.opt);
  s->sim.last_counters = ctr;
  s->sim.fluid_stats = fs;
  if (fstats) to_mg(fs, fstats);
  put(imp.impulses, impulses);
  put_reals(imp.angular_impulses, angular);
  if (clamp_hits) *clamp_hits = imp.clamp_hits;
  if (fluid_momentum) { fluid_momentum[0] = imp.fluid_momentum_change.x; fluid_momentum[1] = imp.fluid_momentum_change.y; }
  return MG_OK;
}

int or_dem_step_recorded(OrSim* s, const MgDrum* drum, float drum_angle, const MgMediaParams* media, uint32_t it,
                         float dt, const float* impulses, const float* angular, MgDemStepStats* dstats,
                         MgImpactRecord* out, uint32_t cap, uint32_t* n_out) {
  Drum d = to_drum(drum);
  MediaParams m;
  std::memcpy(&m, media, sizeof(m));
  size_t nb = s->sim.balls.len();
  CouplingImpulses imp;
  imp.zeros(nb);
  if (impulses) imp.impulses = vecs(impulses, (uint32_t)nb);
  if (angular) imp.angular_impulses.assign(angular, angular + nb);
  std::vector<ImpactRecord> recs;
  StepCounters ctr;
  DemStepStats ds = dem_step_recorded(&s->sim.balls, d, drum_angle, m, it, dt, (impulses || angular) ? &imp : nullptr,
                                      &recs, &ctr, &s->sim.dbg);
  s->sim.last_counters = ctr;  // the DEM half's counters; the fluid ones read 0, as on the device
  s->sim.last_dem_stats = ds;
  if (dstats) to_mg(ds, dstats);
  if (n_out) *n_out = (uint32_t)recs.size();
  if (out)
    for (size_t k = 0; k < recs.size() && k < cap; ++k) std::memcpy(&out[k], &recs[k], sizeof(ImpactRecord));
  return MG_OK;
}

int or_get_counts(const OrSim* s, uint32_t* nb, uint32_t* nf) {
  if (nb) *nb = (uint32_t)s->sim.balls.len();
  if (nf) *nf = (uint32_t)s->sim.fluid.len();
  return MG_OK;
}
int or_get_balls(OrSim* s, float* x, float* v, float* theta, float* omega) {
  const Balls& b = s->sim.balls;
  put(b.x, x);
  put(b.v, v);
  put_reals(b.theta, theta);
  put_reals(b.omega, omega);
  return MG_OK;
}
int or_set_balls(OrSim* s, uint32_t n, const float* x, const float* v, const float* theta, const float* omega) {
  Balls& b = s->sim.balls;
  b.x = vecs(x, n);
  b.v = v ? vecs(v, n) : std::vector<Vec2>(n);
  b.theta = theta ? reals(theta, n) : std::vector<Real>(n, Real(0));
  b.omega = omega ? reals(omega, n) : std::vector<Real>(n, Real(0));
  return MG_OK;
}
int or_get_ball_material(const OrSim* s, MgBallMaterial* o) {
  const Balls& b = s->sim.balls;
  *o = {(float)b.radius, (float)b.mass, (float)b.inertia, (float)b.true_radius};
  return MG_OK;
}
int or_set_ball_material(OrSim* s, const MgBallMaterial* m) {
  Balls& b = s->sim.balls;
  b.radius = m->radius;
  b.mass = m->mass;
  b.inertia = m->inertia;
  b.true_radius = m->true_radius;
  return MG_OK;
}
int or_get_fluid(OrSim* s, float* x, float* v, float* dye, float* guess, uint32_t* guess_len) {
  const Fluid& f = s->sim.fluid;
  put(f.x, x);
  put(f.v, v);
  put_reals(f.dye, dye);
  if (guess_len) *guess_len = (uint32_t)f.viscous_guess.size();
  put(f.viscous_guess, guess);
  return MG_OK;
}
int or_set_fluid(OrSim* s, uint32_t n, const float* x, const float* v, const float* dye, const float* guess) {
  Fluid& f = s->sim.fluid;
  f.x = vecs(x, n);
  f.v = v ? vecs(v, n) : std::vector<Vec2>(n);
  f.dye = dye ? reals(dye, n) : std::vector<Real>(n, Real(0));
  if (guess) f.viscous_guess = vecs(guess, n);
  else f.viscous_guess.clear();
  return MG_OK;
}
int or_get_fluid_material(const OrSim* s, MgFluidMaterial* o) {
  const Fluid& f = s->sim.fluid;
  *o = {(float)f.particle_mass, (float)f.h, (float)f.rest_density};
  return MG_OK;
}
int or_set_fluid_material(OrSim* s, const MgFluidMaterial* m) {
  Fluid& f = s->sim.fluid;
  f.particle_mass = m->particle_mass;
  f.h = m->h;
  f.rest_density = m->rest_density;
  return MG_OK;
}

int or_get_scalars(OrSim* s, MgScalars* o) {
  const Simulation& q = s->sim;
  std::memset(o, 0, sizeof(*o));
  o->drum_angle = q.drum_angle;
  o->power_draw_w = q.power_draw_w;
  o->torque_nm = q.torque_nm;
  o->collision_rate_per_s = q.collision_rate_per_s;
  o->dissipated_power_w = q.dissipated_power_w;
  o->max_substep_displacement_over_diameter = q.max_substep_displacement_over_diameter;
  o->coupling_clamp_hits = q.coupling_clamp_hits;
  o->viscosity_iterations = q.fluid_stats.viscosity_iterations;
  o->mean_shear_rate_per_s = q.fluid_stats.mean_shear_rate_per_s;
  o->sim_time = q.sim_time;
  return MG_OK;
}
int or_energy_budget(OrSim* s, MgEnergyBudget* o) {
  EnergyBudget b = s->sim.energy_budget_now();
  std::memcpy(o, &b, sizeof(b));
  return MG_OK;
}
int or_state_hash(OrSim* s, int ext, uint64_t* out) {
  *out = state_hash(s->sim.balls, s->sim.fluid, ext != 0);
  return MG_OK;
}
int or_metrics(OrSim* s, MgMetrics* out) {
  if (!s || !out) { g_err = "null argument"; return MG_ERR_ARG; }
  metrics_compute(s->sim.balls, s->sim.fluid, s->sim.drum(), s->sim.drum_angle, out);
  return MG_OK;
}
int or_fluid_surface(OrSim* s, float* out, uint32_t cap, uint32_t* len) {
  if (!s || !len) { g_err = "null argument"; return MG_ERR_ARG; }
  const std::vector<Real> flat = surface_extract_flat(s->sim.fluid, s->sim.drum(), s->sim.drum_angle);
  *len = (uint32_t)flat.size();
  if (!out) return MG_OK;
  if (cap < flat.size()) { g_err = "output buffer too small"; return MG_ERR_CAPACITY; }
  put_reals(flat, out);
  return MG_OK;
}
int or_surface_field(OrSim* s, float* field, float* phi_full) {
  if (!s) { g_err = "null argument"; return MG_ERR_ARG; }
  if (field) {
    const std::vector<Real> f = surface_build_field(s->sim.fluid, s->sim.drum(), s->sim.drum_angle);
    put_reals(f, field);
  }
  if (phi_full) *phi_full = surface_phi_full(s->sim.fluid);
  return MG_OK;
}
int or_mixing_index(OrSim* s, float* out, int* valid) {
  Real m = Real(0);
  *valid = mixing_index(s->sim.fluid, s->sim.drum(), &m) ? 1 : 0;
  *out = (float)m;
  return MG_OK;
}
int or_stress_histogram_rate(OrSim* s, double* out) {
  std::copy(s->sim.stress.hist_rate, s->sim.stress.hist_rate + SE_BINS, out);
  return MG_OK;
}
int or_stress_set_debounce_factor(OrSim* s, double f) {
  s->sim.stress.has_debounce = true;
  s->sim.stress.debounce_factor = f;
  return MG_OK;
}
int or_last_step_stats(OrSim* s, MgFluidStepStats* f, MgDemStepStats* d, MgStepCounters* c) {
  if (f) to_mg(s->sim.fluid_stats, f);
  if (d) to_mg(s->sim.last_dem_stats, d);
  if (c) std::memcpy(c, &s->sim.last_counters, sizeof(*c));
  return MG_OK;
}
int or_fluid_densities(OrSim* s, float* out) {
  put_reals(fluid_densities(s->sim.fluid), out);
  return MG_OK;
}
double or_total_mechanical_energy(OrSim* s) { return s->sim.total_mechanical_energy_j(); }

// ---- grid-stage probes
int or_probe_grid(const float* xy, uint32_t n, float cell, int32_t* min_cxy, int64_t* wh, uint32_t* cell_start,
                  uint32_t cell_cap, uint32_t* indices, uint32_t* n_cells_out, int* dense_out) {
  UniformGrid g = UniformGrid::build(vecs(xy, n), cell);
  *dense_out = g.dense ? 1 : 0;
  min_cxy[0] = g.min_cx;
  min_cxy[1] = g.min_cy;
  wh[0] = g.width;
  wh[1] = g.height;
  *n_cells_out = (uint32_t)g.cell_start.size();
  if (g.cell_start.size() > cell_cap) return MG_ERR_CAPACITY;
  std::copy(g.cell_start.begin(), g.cell_start.end(), cell_start);
  std::copy(g.indices.begin(), g.indices.end(), indices);
  return MG_OK;
}
int or_probe_candidate_pairs(const float* xy, uint32_t n, float cell, uint32_t* pairs, uint32_t cap, uint32_t* n_out) {
  auto p = candidate_pairs(vecs(xy, n), cell);
  *n_out = (uint32_t)p.size();
  if (p.size() > cap) return MG_ERR_CAPACITY;
  for (size_t k = 0; k < p.size(); ++k) { pairs[2 * k] = p[k].first; pairs[2 * k + 1] = p[k].second; }
  return MG_OK;
}
int or_probe_neighbor_lists(const float* xy, uint32_t n, float h, uint32_t* offsets, uint32_t* nbrs, uint32_t cap,
                            uint32_t* n_edges) {
  std::vector<uint32_t> off, nb;
  neighbor_lists(vecs(xy, n), h, &off, &nb);
  *n_edges = (uint32_t)nb.size();
  std::copy(off.begin(), off.end(), offsets);
  if (nb.size() > cap) return MG_ERR_CAPACITY;
  std::copy(nb.begin(), nb.end(), nbrs);
  return MG_OK;
}
int or_probe_near(const float* xy, uint32_t n, float cell, float px, float py, uint32_t* out, uint32_t cap,
                  uint32_t* n_out) {
  UniformGrid g = UniformGrid::build(vecs(xy, n), cell);
  std::vector<uint32_t> r;
  g.for_each_near(Vec2(px, py), [&](uint32_t i) { r.push_back(i); });
  *n_out = (uint32_t)r.size();
  for (size_t k = 0; k < r.size() && k < cap; ++k) out[k] = r[k];
  return MG_OK;
}
int or_last_neighbor_lists(OrSim* s, uint32_t* offsets, uint32_t* nbrs, uint32_t cap, uint32_t* n_edges) {
  const Debug& d = s->sim.dbg;
  *n_edges = (uint32_t)d.nbrs.size();
  std::copy(d.nbr_offsets.begin(), d.nbr_offsets.end(), offsets);
  if (d.nbrs.size() > cap) return MG_ERR_CAPACITY;
  std::copy(d.nbrs.begin(), d.nbrs.end(), nbrs);
  return MG_OK;
}
int or_last_ball_pairs(OrSim* s, uint32_t* pairs, uint32_t cap, uint32_t* n_out) {
  const Debug& d = s->sim.dbg;
  *n_out = (uint32_t)d.ball_pairs.size();
  if (d.ball_pairs.size() > cap) return MG_ERR_CAPACITY;
  for (size_t k = 0; k < d.ball_pairs.size(); ++k) {
    pairs[2 * k] = d.ball_pairs[k].first;
    pairs[2 * k + 1] = d.ball_pairs[k].second;
  }
  return MG_OK;
}

// ---- scalar helpers the reference's unit tests exercise
void or_sdf_world(const MgDrum* drum, float px, float py, float angle, float* d, float* nx, float* ny) {
  Vec2 n;
  Real dd;
  to_drum(drum).sdf_world(Vec2(px, py), angle, &dd, &n);
  *d = (float)dd;
  *nx = (float)n.x;
  *ny = (float)n.y;
}
float or_sdf_local(const MgDrum* drum, float px, float py) { return to_drum(drum).sdf(Vec2(px, py)); }
int or_toi_swept(const MgDrum* drum, float x0, float y0, float x1, float y1, float a0, float a1, float radius,
                 float* t) {
  Real tt = (Real)*t;  // left as the caller gave it unless the function writes it
  const int hit = to_drum(drum).toi_swept(Vec2(x0, y0), Vec2(x1, y1), a0, a1, radius, &tt) ? 1 : 0;
  *t = (float)tt;
  return hit;
}
float or_effective_friction(float mk, float ms, float vt, float vs) { return effective_friction(mk, ms, vt, vs); }
int or_impact_energy_bin(float e) { return impact_energy_bin(e); }
uint64_t or_rng_next_u64(uint64_t* state) {
  Rng r(1);
  r.state = *state;
  uint64_t v = r.next_u64();
  *state = r.state;
  return v;
}
uint64_t or_rng_seed_state(uint64_t seed) { return Rng(seed).state; }
float or_rng_next_f32(uint64_t* state) {
  Rng r(1);
  r.state = *state;
  float v = r.next_f32();
  *state = r.state;
  return v;
}
int or_se_bin(double e) { return se_bin(e); }

}  // extern "C"

// ---------------------------------------------------------------- stress metrics, seed sweeps
namespace {

const double THRESHOLDS_REL[6] = {0.03, 0.1, 0.3, 1.0, 3.0, 10.0};  // stress.rs:42

// StressAccum::metrics (stress.rs:186-237) with Simulation::metrics's arguments (lib.rs:383-390)
MgStressMetrics stress_metrics(const Simulation& sim) {
  double m3, scale_j, d;
  sim.stress_scales(&m3, &scale_j, &d);
  const StressAccum& st = sim.stress;
  const double n = (double)std::max<size_t>(sim.balls.len(), 1);
  const double power_draw_w = (double)sim.power_draw_w;
  MgStressMetrics o;
  std::memset(&o, 0, sizeof(o));
  for (int c = 0; c < 4; ++c) {
    o.impacts_per_ball_per_s[c] = (float)(st.count_rate[c] / n);
    if (st.count_rate[c] > 0.0) o.mean_se_scaled[c] = (float)(st.se_hat_rate[c] / st.count_rate[c]);
  }
  auto pooled = [&](int a, int b) {
    double w = st.count_rate[a] + st.count_rate[b];
    return w > 0.0 ? (float)((st.se_hat_rate[a] + st.se_hat_rate[b]) / w) : 0.0f;
  };
  const double total = st.total_rate();
  const double power_per_ball = power_draw_w * d / n;
  o.ball_mass_3d_kg = (float)m3;
  o.scale_energy_j = (float)scale_j;
  o.impacts_total_per_ball_per_s = (float)(total / n);
  o.mean_se_scaled_drop = pooled(0, 2);
  o.mean_se_scaled_shear = pooled(1, 3);
  double se_sum = 0.0;
  for (int c = 0; c < 4; ++c) se_sum += st.se_hat_rate[c];
  o.stress_intensity_scaled = total > 0.0 ? (float)(se_sum / total) : 0.0f;
  o.wall_power_per_ball_w = (float)power_per_ball;
  o.specific_power_w_per_kg = (float)(power_per_ball / m3);
  for (int q = 0; q < 6; ++q) {
    o.thresholds_scaled[q] = (float)THRESHOLDS_REL[q];
    o.effective_power_per_ball_w[q] = (float)(st.above_rate_j[q] / n);
    o.cumulative_effective_energy_per_ball_j[q] = st.cum_above_j[q] / n;
  }
  o.cumulative_wall_energy_per_ball_j = st.cum_wall_j * d / n;
  o.cumulative_specific_energy_j_per_kg = st.cum_wall_j * d / n / m3;
  return o;
}

// batch.rs:126-139 values(): the 16 per-frame scalars in name order
void frame_values(const MgStressMetrics& m, double* v) {
  v[0] = m.specific_power_w_per_kg;
  v[1] = m.wall_power_per_ball_w;
  v[2] = m.impacts_total_per_ball_per_s;
  v[3] = m.mean_se_scaled_drop;
  v[4] = m.mean_se_scaled_shear;
  v[5] = m.stress_intensity_scaled;
  for (int c = 0; c < 4; ++c) v[6 + c] = m.impacts_per_ball_per_s[c];
  for (int q = 0; q < 6; ++q) v[10 + q] = m.effective_power_per_ball_w[q];
}

// batch.rs:141-159
double drift_per_rev(const double* y, size_t len, double frames_per_rev) {
  if (len < 2) return 0.0;
  const double n = (double)len;
  double sum = 0.0;
  for (size_t i = 0; i < len; ++i) sum += y[i];
  const double mean = sum / n, xm = (n - 1.0) / 2.0;
  double sxy = 0.0, sxx = 0.0;
  for (size_t i = 0; i < len; ++i) {
    sxy += ((double)i - xm) * (y[i] - mean);
    sxx += ((double)i - xm) * ((double)i - xm);
  }
  return std::fabs(mean) > 0.0 && sxx > 0.0 ? sxy / sxx * frames_per_rev / std::fabs(mean) : 0.0;
}

const char* const SEED_VALUE_NAMES[MG_SEED_VALUES] = {
    "specific_power_w_per_kg", "wall_power_per_ball_w", "impacts_total_per_ball_per_s", "mean_se_scaled_drop",
    "mean_se_scaled_shear", "stress_intensity_scaled", "impacts_per_ball_per_s.ball_ball_drop",
    "impacts_per_ball_per_s.ball_ball_shear", "impacts_per_ball_per_s.ball_wall_drop",
    "impacts_per_ball_per_s.ball_wall_shear", "effective_power_per_ball_w.thr0", "effective_power_per_ball_w.thr1",
    "effective_power_per_ball_w.thr2", "effective_power_per_ball_w.thr3", "effective_power_per_ball_w.thr4",
    "effective_power_per_ball_w.thr5", "window_specific_power_w_per_kg", "window_effective_power_per_ball_w.thr0",
    "window_effective_power_per_ball_w.thr1", "window_effective_power_per_ball_w.thr2",
    "window_effective_power_per_ball_w.thr3", "window_effective_power_per_ball_w.thr4",
    "window_effective_power_per_ball_w.thr5"};

// batch.rs:40-107 run_seed
int run_seed(const Params& params, uint64_t seed, float warmup_revolutions, float measure_revolutions,
             MgSeedResult* out) {
  Params p = params;
  p.simulation.seed = seed;
  const double omega = (double)(mill_rpm(p.mill) * 2.0f * PI_F / 60.0f);
  if (omega <= 1e-6) { g_err = "mill speed must be > 0"; return MG_ERR_ARG; }
  if (!(measure_revolutions >= 1.0f && warmup_revolutions >= 0.0f)) {
    g_err = "measure_revolutions must be >= 1 and warmup_revolutions >= 0";
    return MG_ERR_ARG;
  }
  const double rev_s = 6.283185307179586 / omega;
  Simulation sim;
  std::string e;
  if (!Simulation::build(p, nullptr, &sim, &e)) { g_err = e; return MG_ERR_INVALID_PARAMS; }
  const size_t warm = (size_t)std::round((double)warmup_revolutions * rev_s * 60.0);
  const size_t meas = (size_t)std::max(std::round((double)measure_revolutions * rev_s * 60.0), 1.0);
  const float frame_s = 1.0f / 60.0f;
  for (size_t f = 0; f < warm; ++f) sim.step(frame_s);
  const MgStressMetrics start = stress_metrics(sim);
  double sum[16] = {};
  std::vector<double> powers;
  powers.reserve(meas);
  for (size_t f = 0; f < meas; ++f) {
    sim.step(frame_s);
    const MgStressMetrics m = stress_metrics(sim);
    double v[16];
    frame_values(m, v);
    for (int k = 0; k < 16; ++k) sum[k] += v[k];
    powers.push_back((double)m.wall_power_per_ball_w);
  }
  const MgStressMetrics end = stress_metrics(sim);
  const double n = (double)meas, window_s = n * (double)frame_s;
  std::memset(out, 0, sizeof(*out));
  out->seed = seed;
  out->window_s = window_s;
  out->coarse_graining_factor = effective_media(p).scale_factor;
  for (int k = 0; k < 16; ++k) out->values[k] = sum[k] / n;
  out->values[16] = (end.cumulative_specific_energy_j_per_kg - start.cumulative_specific_energy_j_per_kg) / window_s;
  for (int q = 0; q < 6; ++q)
    out->values[17 + q] =
        (end.cumulative_effective_energy_per_ball_j[q] - start.cumulative_effective_energy_per_ball_j[q]) / window_s;
  out->power_drift_rel_per_rev = drift_per_rev(powers.data(), powers.size(), rev_s * 60.0);
  return MG_OK;
}

}  // namespace

extern "C" {

int or_stress_metrics(OrSim* s, MgStressMetrics* out) {
  if (!s || !out) { g_err = "null argument"; return MG_ERR_ARG; }
  *out = stress_metrics(s->sim);
  return MG_OK;
}
const char* or_seed_value_name(uint32_t k) { return k < MG_SEED_VALUES ? SEED_VALUE_NAMES[k] : ""; }
int or_seed_sweep(const MgParams* params, const uint64_t* seeds, uint32_t n_seeds, float warmup_revolutions,
                  float measure_revolutions, MgSeedResult* out) {
  if (!params || (n_seeds && (!seeds || !out))) { g_err = "null argument"; return MG_ERR_ARG; }
  for (uint32_t i = 0; i < n_seeds; ++i) {
    int rc = run_seed(to_p(params), seeds[i], warmup_revolutions, measure_revolutions, &out[i]);
    if (rc) return rc;
  }
  return MG_OK;
}
// batch.rs:161-190 combine
int or_seed_combine(const MgSeedResult* r, uint32_t n, double* mean, double* std_err) {
  if (n == 0) { g_err = "no results to combine"; return MG_ERR_ARG; }
  if (!r || !mean || !std_err) { g_err = "null argument"; return MG_ERR_ARG; }
  const double nn = (double)n;
  for (int k = 0; k < MG_SEED_VALUES; ++k) {
    double s = 0.0;
    for (uint32_t i = 0; i < n; ++i) s += r[i].values[k];
    const double m = s / nn;
    double se = 0.0;
    if (n >= 2) {
      double v = 0.0;
      for (uint32_t i = 0; i < n; ++i) { double dv = r[i].values[k] - m; v += dv * dv; }
      se = std::sqrt(v / (nn - 1.0) / nn);
    }
    mean[k] = m;
    std_err[k] = se;
  }
  return MG_OK;
}
double or_seed_drift_per_rev(const double* y, uint32_t n, double frames_per_rev) {
  return drift_per_rev(y, n, frames_per_rev);
}

}  // extern "C"
