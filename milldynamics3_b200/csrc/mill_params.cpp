// Host-side Params logic and seeding of the library (see mill_params.h for the references).
#include "mill_params.h"

#include <algorithm>
#include <cstring>

namespace mgh {

MgParams params_default() {
  MgParams p;
  std::memset(&p, 0, sizeof(p));
  p.mill = {0.063f, MG_SPEED_RPM, 100.0f, MG_DIR_CCW};
  p.media = {0.002f, 0.50f, 0.82f, 6000.0f, 0.7f, 0.5f, 0.25f, 0.35f, 0.25f, 0.35f, 0.02f, 0.01f};
  p.slurry = {1u, 0.35f, 1000.0f, 0.001f, MG_RHEOLOGY_NEWTONIAN, 0.0f, 1.0f, 1.0f, 0.6f, 0.072f, MG_DYE_LEFT_RIGHT};
  p.lifters = {0u, 0.020f, 0.030f, 0.020f, 0.0f};
  p.simulation.resolution = 40;
  p.simulation.substeps = 8;
  p.simulation.pbf_iterations = 3;
  p.simulation.dem_iterations = 2;
  p.simulation.time_scale = 1.0f;
  p.simulation.frame_budget_ms = 12.0f;
  p.simulation.max_balls = 600;
  p.simulation.seed = 1;
  p.simulation.coarse_graining_mode = MG_CG_OFF;
  p.simulation.coarse_graining_k = 1.0f;
  return p;
}

static bool rng01(float x, float lo, float hi) { return x >= lo && x <= hi; }

bool params_validate(const MgParams& p, std::string* err) {
  auto bad = [&](const char* m) { if (err) *err = m; return false; };
  if (!(p.mill.diameter_m > 0.02f && p.mill.diameter_m < 20.0f)) return bad("mill.diameter_m must be in (0.02, 20.0)");
  if (!(std::isfinite(p.mill.speed_value) && p.mill.speed_value >= 0.0f)) return bad("mill.speed_value must be finite and >= 0");
  if (p.mill.speed_mode > 1 || p.mill.direction > 1) return bad("mill enum out of range");
  const MgMediaParams& d = p.media;
  if (!(d.ball_diameter_m > 0.0005f && d.ball_diameter_m < 1.0f)) return bad("media.ball_diameter_m must be in (0.0005, 1.0)");
  if (!rng01(d.fill_fraction, 0.0f, 0.9f)) return bad("media.fill_fraction must be in [0, 0.9]");
  if (!rng01(d.packing_fraction_2d, 0.5f, 0.907f)) return bad("media.packing_fraction_2d must be in [0.5, 0.907]");
  if (!(std::isfinite(d.density_kg_m3) && d.density_kg_m3 > 0.0f)) return bad("media.density_kg_m3 must be > 0");
  if (!rng01(d.restitution_ball_ball, 0.0f, 1.0f)) return bad("media.restitution_ball_ball must be in [0, 1]");
  if (!rng01(d.restitution_ball_wall, 0.0f, 1.0f)) return bad("media.restitution_ball_wall must be in [0, 1]");
  const float mus[5] = {d.friction_ball_ball, d.friction_ball_wall, d.friction_ball_ball_static,
                        d.friction_ball_wall_static, d.rolling_friction};
  const char* names[5] = {"media.friction_ball_ball must be >= 0", "media.friction_ball_wall must be >= 0",
                          "media.friction_ball_ball_static must be >= 0", "media.friction_ball_wall_static must be >= 0",
                          "media.rolling_friction must be >= 0"};
  for (int k = 0; k < 5; ++k)
    if (!(mus[k] >= 0.0f && std::isfinite(mus[k]))) return bad(names[k]);
  if (d.friction_ball_ball_static < d.friction_ball_ball) return bad("media.friction_ball_ball_static must be >= media.friction_ball_ball");
  if (d.friction_ball_wall_static < d.friction_ball_wall) return bad("media.friction_ball_wall_static must be >= media.friction_ball_wall");
  if (!(d.friction_velocity_scale_m_s > 0.0f && std::isfinite(d.friction_velocity_scale_m_s))) return bad("media.friction_velocity_scale_m_s must be > 0");
  const MgSlurryParams& s = p.slurry;
  if (!rng01(s.fill_fraction, 0.0f, 0.9f)) return bad("slurry.fill_fraction must be in [0, 0.9]");
  if (!(std::isfinite(s.density_kg_m3) && s.density_kg_m3 > 0.0f)) return bad("slurry.density_kg_m3 must be > 0");
  if (!(s.viscosity_pa_s >= 0.0f && std::isfinite(s.viscosity_pa_s))) return bad("slurry.viscosity_pa_s must be >= 0");
  if (!(s.yield_stress_pa >= 0.0f && std::isfinite(s.yield_stress_pa))) return bad("slurry.yield_stress_pa must be >= 0");
  if (!(s.surface_tension_n_m >= 0.0f && std::isfinite(s.surface_tension_n_m))) return bad("slurry.surface_tension_n_m must be >= 0");
  if (!rng01(s.wall_no_slip, 0.0f, 1.0f)) return bad("slurry.wall_no_slip must be in [0, 1]");
  if (!rng01(s.ball_no_slip, 0.0f, 1.0f)) return bad("slurry.ball_no_slip must be in [0, 1]");
  if (!rng01(s.wettability, 0.0f, 1.0f)) return bad("slurry.wettability must be in [0, 1]");
  if (s.rheology > 1 || s.dye_pattern > 2) return bad("slurry enum out of range");
  const MgLiftersParams& l = p.lifters;
  if (l.count > 0) {
    if (!(l.height_m > 0.0f && std::isfinite(l.height_m))) return bad("lifters.height_m must be > 0");
    if (!(l.base_width_m > 0.0f && std::isfinite(l.base_width_m))) return bad("lifters.base_width_m must be > 0");
    if (!(l.top_width_m >= 0.0f && std::isfinite(l.top_width_m))) return bad("lifters.top_width_m must be >= 0");
  }
  const MgSimulationParams& q = p.simulation;
  if (!(q.resolution >= 4 && q.resolution <= 200)) return bad("simulation.resolution must be in [4, 200]");
  if (!(q.substeps >= 1 && q.substeps <= 64)) return bad("simulation.substeps must be in [1, 64]");
  if (!(q.pbf_iterations >= 1 && q.pbf_iterations <= 20)) return bad("simulation.pbf_iterations must be in [1, 20]");
  if (!(q.dem_iterations >= 1 && q.dem_iterations <= 20)) return bad("simulation.dem_iterations must be in [1, 20]");
  if (!(q.time_scale > 0.0f && std::isfinite(q.time_scale))) return bad("simulation.time_scale must be > 0");
  if (!(q.frame_budget_ms > 0.0f && std::isfinite(q.frame_budget_ms))) return bad("simulation.frame_budget_ms must be > 0");
  if (!(q.max_balls >= 10 && q.max_balls <= 50000)) return bad("simulation.max_balls must be in [10, 50000]");
  if (!(q.coarse_graining_k >= 1.0f && q.coarse_graining_k <= 1000.0f)) return bad("simulation.coarse_graining_k must be in [1, 1000]");
  if (q.coarse_graining_mode > 2) return bad("simulation enum out of range");
  if (l.count > 64) return bad("lifters.count above the supported 64");
  return true;
}

bool preset_apply(MgParams* p, const char* id) {
  std::string s(id ? id : "");
  if (s == "realtime") { p->simulation.max_balls = 300; p->simulation.resolution = 25; return true; }
  if (s == "balanced") { p->simulation.max_balls = 300; p->simulation.resolution = 30; return true; }
  if (s == "accuracy") { p->simulation.max_balls = 600; p->simulation.resolution = 50; return true; }
  if (s == "impact_stats") {
    p->simulation.max_balls = 600;
    p->simulation.resolution = 25;
    p->simulation.substeps = 32;
    p->simulation.dem_iterations = 12;
    p->simulation.coarse_graining_mode = MG_CG_OFF;
    return true;
  }
  return false;
}

float critical_speed_rpm(const MgMillParams& m) { return 42.3f / std::sqrt(m.diameter_m); }
float mill_rpm(const MgMillParams& m) {
  return m.speed_mode == MG_SPEED_RPM ? m.speed_value : critical_speed_rpm(m) * m.speed_value / 100.0f;
}
float mill_percent_critical(const MgMillParams& m) {
  return m.speed_mode == MG_SPEED_PERCENT_CRITICAL ? m.speed_value : 100.0f * m.speed_value / critical_speed_rpm(m);
}
float mill_omega(const MgMillParams& m) {
  float w = mill_rpm(m) * 2.0f * PI_F / 60.0f;
  return m.direction == MG_DIR_CCW ? w : -w;
}
float true_ball_count(const MgParams& p) {
  float r_true = p.media.ball_diameter_m * 0.5f;
  if (r_true <= 0.0f) return 0.0f;
  float rr = mill_radius(p.mill);
  float area = PI_F * (rr * rr);
  return (p.media.fill_fraction * p.media.packing_fraction_2d * area) / (PI_F * r_true * r_true);
}
Effective effective_media(const MgParams& p) {
  float true_d = p.media.ball_diameter_m;
  float n_true = true_ball_count(p);
  float max_balls = (float)p.simulation.max_balls;
  float k = 1.0f;
  if (p.simulation.coarse_graining_mode == MG_CG_MANUAL) k = fmax_r(p.simulation.coarse_graining_k, 1.0f);
  else if (p.simulation.coarse_graining_mode == MG_CG_AUTO)
    k = (n_true > max_balls && max_balls > 0.0f) ? std::sqrt(n_true / max_balls) : 1.0f;
  if (k > 1.0f) return {true_d, true_d * k, p.media.density_kg_m3, f2u_sat(fmax_r(std::round(n_true / (k * k)), 1.0f)), k};
  return {true_d, true_d, p.media.density_kg_m3, f2u_sat(fmax_r(std::round(n_true), 0.0f)), 1.0f};
}
uint32_t effective_fluid_resolution(const MgParams& p) {
  float radius = mill_radius(p.mill);
  float d_eff = effective_media(p).diameter_m;
  if (!(radius > 0.0f && d_eff > 0.0f)) return p.simulation.resolution;
  uint32_t mr = f2u_sat(std::ceil(radius / d_eff));
  return std::min(std::max(p.simulation.resolution, mr), 200u);
}
uint32_t effective_substeps(const MgParams& p) {
  float d_eff = effective_media(p).diameter_m;
  float dia = p.mill.diameter_m;
  if (!(d_eff > 0.0f && dia > 0.0f)) return p.simulation.substeps;
  float df = clamp_r(1.0f + 2.5f * (p.media.fill_fraction - 0.30f), 1.0f, 2.0f);
  float v_ref = std::sqrt(2.0f * 9.81f * dia);
  uint32_t mn = f2u_sat(fmax_r(std::ceil(v_ref * df / (60.0f * 0.5f * d_eff)), 1.0f));
  uint32_t cap = f2u_sat(std::ceil(16.0f * df));
  return std::max(p.simulation.substeps, std::min(mn, cap));
}

namespace {
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed == 0 ? 0x9E3779B97F4A7C15ull : seed) {}
  uint64_t next() {
    uint64_t x = s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    s = x;
    return x * 0x2545F4914F6CDD1Dull;
  }
  float f32() { return (float)(next() >> 40) / (float)(1u << 24); }
  float range(float lo, float hi) { return lo + f32() * (hi - lo); }
};
}  // namespace

float ball_mass(float d, float rho) {
  float r = d * 0.5f;
  return rho * PI_F * r * r;
}

void seed_balls(Balls* b, const Effective& e, float drum_r, uint64_t seed) {
  float r = e.diameter_m * 0.5f;
  float mass = ball_mass(e.diameter_m, e.density_kg_m3);
  size_t count = e.ball_count;
  Rng rng(seed);
  std::vector<float> x;
  if (r > 0.0f && count > 0) {
    float spacing = 2.0f * r * 1.02f;
    float row_h = spacing * (std::sqrt(3.0f) * 0.5f);
    float fill_r = fmax_r(drum_r - r, 0.0f);
    int32_t n_rows = f2i_sat(std::ceil(2.0f * fill_r / row_h)) + 1;
    for (int32_t row = -n_rows / 2; row <= n_rows / 2 && x.size() / 2 < count; ++row) {
      float y = (float)row * row_h;
      if (std::fabs(y) > fill_r) continue;
      float hw = std::sqrt(fmax_r(fill_r * fill_r - y * y, 0.0f));
      float off = (((row % 2) + 2) % 2 == 0) ? 0.0f : spacing * 0.5f;
      int32_t n_cols = f2i_sat(std::floor(2.0f * hw / spacing));
      for (int32_t col = -n_cols / 2; col <= n_cols / 2; ++col) {
        float cx = (float)col * spacing + off;
        if (cx * cx + y * y > fill_r * fill_r) continue;
        float jx = rng.range(-0.05f, 0.05f);
        float jy = rng.range(-0.05f, 0.05f);
        x.push_back(cx + jx * r);
        x.push_back(y + jy * r);
        if (x.size() / 2 >= count) break;
      }
    }
  }
  size_t n = x.size() / 2;
  b->x = x;
  b->v.assign(2 * n, 0.0f);
  b->theta.assign(n, 0.0f);
  b->omega.assign(n, 0.0f);
  b->radius = r;
  b->mass = mass;
  b->inertia = 0.5f * mass * r * r;
  b->true_radius = e.true_diameter_m * 0.5f;
}

void seed_fluid(Fluid* f, const MgSlurryParams& s, float drum_r, uint32_t res, const std::vector<float>& bxy,
                float ball_r) {
  float dx = drum_r / (float)std::max(res, 1u);
  float h = 2.0f * dx;
  float row_h = dx * (std::sqrt(3.0f) * 0.5f);
  float cell_area = dx * row_h;
  float target_area = s.fill_fraction * PI_F * drum_r * drum_r;
  size_t target = f2u_sat(fmax_r(std::round(target_area / cell_area), 0.0f));
  std::vector<float> x, dye;
  size_t nb = bxy.size() / 2;
  if (target > 0 && dx > 0.0f) {
    int32_t n_rows = f2i_sat(std::ceil(2.0f * drum_r / row_h)) + 1;
    for (int32_t row = -n_rows / 2; row <= n_rows / 2 && dye.size() < target; ++row) {
      float y = (float)row * row_h;
      if (std::fabs(y) > drum_r) continue;
      float hw = std::sqrt(fmax_r(drum_r * drum_r - y * y, 0.0f));
      float off = (((row % 2) + 2) % 2 == 0) ? 0.0f : dx * 0.5f;
      int32_t n_cols = f2i_sat(std::floor(2.0f * hw / dx));
      for (int32_t col = -n_cols / 2; col <= n_cols / 2; ++col) {
        float cx = (float)col * dx + off;
        if (cx * cx + y * y > drum_r * drum_r) continue;
        bool hit = false;
        for (size_t b = 0; b < nb && !hit; ++b) {
          float ddx = cx - bxy[2 * b], ddy = y - bxy[2 * b + 1];
          hit = std::sqrt(ddx * ddx + ddy * ddy) < ball_r;
        }
        if (hit) continue;
        float dv = 0.0f;
        if (s.dye_pattern == MG_DYE_LEFT_RIGHT) dv = cx < 0.0f ? 0.0f : 1.0f;
        else if (s.dye_pattern == MG_DYE_TOP_BOTTOM) dv = y < 0.0f ? 0.0f : 1.0f;
        dye.push_back(dv);
        x.push_back(cx);
        x.push_back(y);
        if (dye.size() >= target) break;
      }
    }
  }
  f->x = x;
  f->v.assign(x.size(), 0.0f);
  f->dye = dye;
  f->guess.clear();
  f->particle_mass = s.density_kg_m3 * cell_area;
  f->h = h;
  f->rest_density = s.density_kg_m3;
}

double balls_energy_f64(const Balls& b) {
  double e = 0.0;
  for (size_t i = 0; i < b.len(); ++i) {
    float vx = b.v[2 * i], vy = b.v[2 * i + 1];
    e += 0.5 * (double)b.mass * (double)((vx * vx) + (vy * vy));
    e += 0.5 * (double)b.inertia * (double)(b.omega[i] * b.omega[i]);
    e += (double)b.mass * (double)9.81f * (double)b.x[2 * i + 1];
  }
  return e;
}
double fluid_energy_f64(const Fluid& f) {
  double py = 0.0, ke = 0.0;
  for (size_t i = 0; i < f.len(); ++i) py += (double)f.x[2 * i + 1];
  for (size_t i = 0; i < f.len(); ++i) {
    float vx = f.v[2 * i], vy = f.v[2 * i + 1];
    ke += (double)((vx * vx) + (vy * vy));
  }
  return 0.5 * (double)f.particle_mass * ke + py * (double)f.particle_mass * (double)9.81f;
}

}  // namespace mgh
