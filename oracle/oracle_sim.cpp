// Oracle (test infrastructure only): lib.rs Simulation (build, step, advance_one_sub_step,
// update_grinding_stats, energy budget), stress.rs StressAccum::update, metrics.rs mixing_index,
// and the FNV-1a state hash of examples/perf_probe.rs:230-262.
#include <algorithm>
#include <cstring>

#include "oracle_core.hpp"

namespace orc {

// ------------------------------------------------------------------ stress.rs:28-171
static const double SE_BINS_PER_DECADE = 4.0;
static const double SE_LOG10_MIN = -3.0;
static const double THRESHOLDS_REL[6] = {0.03, 0.1, 0.3, 1.0, 3.0, 10.0};

int se_bin(double e_hat) {
  if (std::isnan(e_hat) || e_hat <= 0.0) return 0;
  double t = (std::log10(e_hat) - SE_LOG10_MIN) * SE_BINS_PER_DECADE;
  uint64_t idx = d2u64_sat(dmax_r(t, 0.0));
  return (int)std::min<uint64_t>(idx, SE_BINS - 1);
}

static void classify(const ImpactRecord& rec, double m3, int* cls, double* se) {
  bool bb = rec.kind == 0;
  double vn = (double)rec.normal_speed, vs = (double)rec.slip_speed;
  bool shear = vs > vn;
  *cls = bb ? (shear ? 1 : 0) : (shear ? 3 : 2);
  double m_red = bb ? 0.5 * m3 : m3;
  *se = 0.5 * m_red * (vn * vn + vs * vs);
}

void StressAccum::update(const std::vector<ImpactRecord>& recs, double m3, double scale_j, double d, double now_s,
                         double sub_dt, double alpha, double wall_work_j) {
  double window = (has_debounce ? debounce_factor : 0.25) * std::sqrt(d / 9.81);
  updates += 1;
  if (updates % 4096 == 0) {
    for (auto it = last_counted.begin(); it != last_counted.end();) {
      if (!(now_s - it->second < 4.0 * window)) it = last_counted.erase(it);
      else ++it;
    }
  }
  double count[4] = {}, se_hat[4] = {}, hist[SE_BINS] = {}, above[6] = {};
  for (const ImpactRecord& rec : recs) {
    if (window > 0.0) {
      std::pair<uint32_t, uint32_t> key = {std::min(rec.ball, rec.partner), std::max(rec.ball, rec.partner)};
      if (rec.partner == WALL_ID) key = {rec.ball, WALL_ID};
      auto it = last_counted.find(key);
      if (it != last_counted.end() && now_s - it->second < window) continue;
      last_counted[key] = now_s;
    }
    int cls;
    double se;
    classify(rec, m3, &cls, &se);
    double e_hat = se / scale_j;
    count[cls] += 1.0;
    se_hat[cls] += e_hat;
    hist[se_bin(e_hat)] += 1.0;
    for (int q = 0; q < 6; ++q)
      if (e_hat >= THRESHOLDS_REL[q]) above[q] += se;
  }
  cum_wall_j += wall_work_j;
  for (int q = 0; q < 6; ++q) cum_above_j[q] += above[q];
  auto ema = [&](double* s, double inst) { *s += alpha * (inst / sub_dt - *s); };
  for (int c = 0; c < 4; ++c) { ema(&count_rate[c], count[c]); ema(&se_hat_rate[c], se_hat[c]); }
  for (int b = 0; b < SE_BINS; ++b) ema(&hist_rate[b], hist[b]);
  for (int q = 0; q < 6; ++q) ema(&above_rate_j[q], above[q]);
}

// ------------------------------------------------------------------ lib.rs:138-204
bool Simulation::build(const Params& p, const std::vector<Vec2>* initial, Simulation* s, std::string* err) {
  if (!params_validate(p, err)) return false;
  Real radius = mill_radius(p.mill);
  EffectiveMedia eff = effective_media(p);
  s->params = p;
  balls_seed_lattice(&s->balls, eff, radius, p.simulation.seed);
  if (initial) {
    size_t n = initial->size();
    s->balls.x = *initial;
    s->balls.v.assign(n, Vec2());
    s->balls.theta.assign(n, Real(0.0));
    s->balls.omega.assign(n, Real(0.0));
  }
  uint32_t res = effective_fluid_resolution(p);
  if (p.slurry.enabled) {
    fluid_seed_lattice(&s->fluid, p.slurry, radius, res, s->balls.x, s->balls.radius);
  } else {
    SlurryParams sp = p.slurry;
    sp.fill_fraction = Real(0.0);
    fluid_seed_lattice(&s->fluid, sp, radius, res, std::vector<Vec2>(), Real(0.0));
  }
  if (initial) {
    Real w = mill_omega(p.mill);
    for (size_t i = 0; i < s->balls.len(); ++i) s->balls.v[i] = w * Vec2(-s->balls.x[i].y, s->balls.x[i].x);
    for (size_t i = 0; i < s->balls.len(); ++i) s->balls.omega[i] = w;
    for (size_t i = 0; i < s->fluid.len(); ++i) s->fluid.v[i] = w * Vec2(-s->fluid.x[i].y, s->fluid.x[i].x);
  }
  s->energy_budget_e0 = dem_mechanical_energy_f64(s->balls) + fluid_mechanical_energy(s->fluid);
  s->drum_angle = Real(0.0);
  s->sim_time = 0.0;
  return true;
}

double Simulation::total_mechanical_energy_j() const {
  return dem_mechanical_energy_f64(balls) + fluid_mechanical_energy(fluid);
}

// lib.rs:218-229
EnergyBudget Simulation::energy_budget_now() const {
  EnergyBudget b = energy_budget;
  b.delta_mechanical_j = total_mechanical_energy_j() - energy_budget_e0;
  double explained = b.shaft_work_j - b.ball_contact_dissipation_j - b.fluid_wall_slip_j - b.fluid_viscous_j -
                     b.fluid_clamp_removed_j + b.interface_created_j;
  b.unattributed_j = b.delta_mechanical_j - explained;
  return b;
}

// lib.rs:233-240
void Simulation::stress_scales(double* m3, double* scale_j, double* d) const {
  double r = (double)balls.radius;
  *m3 = (double)balls.mass * 4.0 / 3.0 * r;
  *d = 2.0 * r;
  *scale_j = *m3 * 9.81 * *d;
}

Drum Simulation::drum() const {
  Drum d;
  d.radius_m = mill_radius(params.mill);
  d.omega = mill_omega(params.mill);
  d.lifters = params.lifters;
  return d;
}

// lib.rs:426-464
Real Simulation::fixed_sub_dt() const { return Real(1.0) / (Real(60.0) * (Real)std::max(effective_substeps(params), 1u)); }
void Simulation::reset_frame_stats() {
  max_substep_displacement_over_diameter = Real(0.0);
  coupling_clamp_hits = 0;
}
void Simulation::step_fixed() { advance_one_sub_step(fixed_sub_dt()); }
void Simulation::step(Real dt) {
  uint32_t n = std::max(effective_substeps(params), 1u);
  Real sub_dt = dt / (Real)n;
  reset_frame_stats();
  for (uint32_t k = 0; k < n; ++k) advance_one_sub_step(sub_dt);
}

// lib.rs:470-509
void Simulation::advance_one_sub_step(Real sub_dt) {
  Real omega = mill_omega(params.mill);
  Drum d = drum();
  impact_log.clear();
  CouplingImpulses imp;
  FluidStepStats fs;
  StepCounters ctr;
  fluid_step_coupled(&fluid, d, drum_angle, params.slurry, params.simulation.pbf_iterations, sub_dt, balls, &imp, &fs,
                     &ctr, &dbg, opt);
  DemStepStats ds = dem_step_recorded(&balls, d, drum_angle, params.media, params.simulation.dem_iterations, sub_dt,
                                      &imp, &impact_log, &ctr, &dbg);
  last_counters = ctr;
  last_dem_stats = ds;
  coupling_clamp_hits += fs.coupling_clamp_hits;
  EnergyBudget& b = energy_budget;
  b.elapsed_s += (double)sub_dt;
  b.dem_wall_work_j += (double)ds.wall_work_j;
  b.fluid_wall_work_j += (double)fs.wall_work_j;
  b.shaft_work_j += (double)(ds.wall_work_j + fs.wall_work_j);
  b.ball_contact_dissipation_j += (double)ds.dissipated_energy_j;
  b.fluid_wall_slip_j += (double)(fs.wall_work_j - fs.ke_delta_noslip_j);
  b.fluid_viscous_j -= (double)fs.ke_delta_viscosity_j;
  b.fluid_clamp_removed_j -= (double)fs.ke_delta_clamp_j;
  b.interface_created_j += (double)(ds.coupling_work_j + fs.ke_delta_drag_j + fs.ke_delta_buoyancy_j);
  b.fluid_wall_angular_impulse += (double)fs.wall_angular_impulse;
  update_grinding_stats(ds, fs.wall_work_j, sub_dt, omega);
  fluid_stats = fs;
  drum_angle = rem_euclid_r(drum_angle + omega * sub_dt, TAU_F);
  sim_time += (double)sub_dt;
}

// lib.rs:516-565
void Simulation::update_grinding_stats(const DemStepStats& s, Real fluid_wall_work, Real sub_dt, Real omega) {
  Real alpha = Real(1.0) - expf_r(-sub_dt / Real(1.0));
  Real power_instant = (s.wall_work_j + fluid_wall_work) / sub_dt;
  power_draw_w += alpha * (power_instant - power_draw_w);
  Real torque_instant = std::fabs(omega) > Real(1e-6) ? power_instant / omega : Real(0.0);
  torque_nm += alpha * (torque_instant - torque_nm);
  double m3, scale_j, d;
  stress_scales(&m3, &scale_j, &d);
  stress.update(impact_log, m3, scale_j, d, sim_time, (double)sub_dt, (double)alpha,
                (double)(s.wall_work_j + fluid_wall_work));
  collision_rate_per_s = (Real)stress.total_rate();
  Real dissipated_instant = fmax_r(s.dissipated_energy_j, Real(0.0)) / sub_dt;
  dissipated_power_w += alpha * (dissipated_instant - dissipated_power_w);
  max_substep_displacement_over_diameter =
      fmax_r(max_substep_displacement_over_diameter, s.max_substep_displacement_over_diameter);
}

// ------------------------------------------------------------------ metrics.rs:506-576
bool mixing_index(const Fluid& f, const Drum& d, Real* out) {
  const int G = 16;
  size_t n = f.len();
  if (n == 0 || d.radius_m <= Real(0.0)) return false;
  Real r = d.radius_m;
  Real cell = Real(2.0) * r / (Real)G;
  Real dye_sum[G * G] = {};
  uint32_t count[G * G] = {};
  Real total_dye = Real(0.0);
  for (size_t i = 0; i < n; ++i) {
    Vec2 p = f.x[i];
    int32_t gi = std::min(std::max(f2i_sat(std::floor((p.x + r) / cell)), 0), G - 1);
    int32_t gj = std::min(std::max(f2i_sat(std::floor((p.y + r) / cell)), 0), G - 1);
    int idx = gj * G + gi;
    dye_sum[idx] += f.dye[i];
    count[idx] += 1;
    total_dye += f.dye[i];
  }
  Real p_mean = total_dye / (Real)n;
  std::vector<Real> means;
  std::vector<uint32_t> counts;
  for (int idx = 0; idx < G * G; ++idx)
    if (count[idx] > 0) { means.push_back(dye_sum[idx] / (Real)count[idx]); counts.push_back(count[idx]); }
  if (means.size() < 2) return false;
  uint32_t wsum = 0;
  for (uint32_t c : counts) wsum += c;
  Real weight_sum = (Real)wsum;
  Real ov = Real(0.0);
  for (size_t q = 0; q < means.size(); ++q) {
    Real dm = means[q] - p_mean;
    ov += (Real)counts[q] * (dm * dm);
  }
  Real observed_var = ov / weight_sum;
  Real s0_sq = p_mean * (Real(1.0) - p_mean);
  Real wa = Real(0.0);
  for (uint32_t c : counts) wa += (Real)c * (Real)c;
  Real weighted_avg = wa / weight_sum;
  Real sr_sq = s0_sq / fmax_r(weighted_avg, Real(1.0));
  if (s0_sq < Real(1e-9)) return false;
  Real denom = s0_sq - sr_sq;
  if (std::fabs(denom) < Real(1e-9)) { *out = Real(1.0); return true; }
  Real m = (s0_sq - observed_var) / denom;
  *out = clamp_r(m, Real(0.0), Real(1.0));
  return true;
}

// examples/perf_probe.rs:230-262
uint64_t state_hash(const Balls& b, const Fluid& f, bool extended) {
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&](Real v) {
    uint32_t bits;
    std::memcpy(&bits, &v, 4);
    for (int k = 0; k < 4; ++k) {
      h ^= (uint64_t)((bits >> (8 * k)) & 0xFFu);
      h *= 0x100000001b3ull;
    }
  };
  for (size_t i = 0; i < b.len(); ++i) {
    mix(b.x[i].x); mix(b.x[i].y); mix(b.v[i].x); mix(b.v[i].y); mix(b.omega[i]);
    if (extended) mix(b.theta[i]);
  }
  for (size_t i = 0; i < f.len(); ++i) {
    mix(f.x[i].x); mix(f.x[i].y); mix(f.v[i].x); mix(f.v[i].y);
    if (extended) mix(f.dye[i]);
  }
  return h;
}

}  // namespace orc
