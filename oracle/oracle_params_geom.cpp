// Oracle (test infrastructure only): params.rs, rng/seeding (dem.rs:355-409, pbf.rs:1044-1119),
// grid.rs and geometry.rs restated. See oracle_core.hpp for the arithmetic conventions.
#include <algorithm>
#include <cstring>

#include "oracle_core.hpp"

namespace orc {

// ------------------------------------------------------------------ params.rs:62-77,185-227,
// 351-375,419-428,505-518 (Default impls)
Params params_default() {
  Params p;
  std::memset(&p, 0, sizeof(p));
  p.mill = {0.063f, SPEED_RPM, 100.0f, DIR_CCW};
  p.media = {0.002f, 0.50f, 0.82f, 6000.0f, 0.7f, 0.5f, 0.25f, 0.35f, 0.25f, 0.35f, 0.02f, 0.01f};
  p.slurry.enabled = 1;
  p.slurry.fill_fraction = 0.35f;
  p.slurry.density_kg_m3 = 1000.0f;
  p.slurry.viscosity_pa_s = 0.001f;
  p.slurry.rheology = RHEO_NEWTONIAN;
  p.slurry.yield_stress_pa = 0.0f;
  p.slurry.wall_no_slip = 1.0f;
  p.slurry.ball_no_slip = 1.0f;
  p.slurry.wettability = 0.6f;
  p.slurry.surface_tension_n_m = 0.072f;
  p.slurry.dye_pattern = DYE_LEFT_RIGHT;
  p.lifters = {0, 0.020f, 0.030f, 0.020f, 0.0f};
  p.simulation.resolution = 40;
  p.simulation.substeps = 8;
  p.simulation.pbf_iterations = 3;
  p.simulation.dem_iterations = 2;
  p.simulation.time_scale = 1.0f;
  p.simulation.frame_budget_ms = 12.0f;
  p.simulation.max_balls = 600;
  p.simulation.seed = 1;
  p.simulation.coarse_graining_mode = CG_OFF;
  p.simulation.coarse_graining_k = 1.0f;
  return p;
}

static bool in_range(float x, float lo, float hi) { return x >= lo && x <= hi; }

// params.rs:115-126, 231-278, 379-405, 432-445, 504-530, 545-552
bool params_validate(const Params& p, std::string* err) {
  auto fail = [&](const std::string& m) { if (err) *err = m; return false; };
  const MillParams& m = p.mill;
  if (!(m.diameter_m > 0.02f && m.diameter_m < 20.0f)) return fail("mill.diameter_m must be in (0.02, 20.0)");
  if (!(std::isfinite(m.speed_value) && m.speed_value >= 0.0f)) return fail("mill.speed_value must be finite and >= 0");
  if (m.speed_mode > 1 || m.direction > 1) return fail("mill enum out of range");
  const MediaParams& d = p.media;
  if (!(d.ball_diameter_m > 0.0005f && d.ball_diameter_m < 1.0f)) return fail("media.ball_diameter_m must be in (0.0005, 1.0)");
  if (!in_range(d.fill_fraction, 0.0f, 0.9f)) return fail("media.fill_fraction must be in [0, 0.9]");
  if (!in_range(d.packing_fraction_2d, 0.5f, 0.907f)) return fail("media.packing_fraction_2d must be in [0.5, 0.907]");
  if (!(std::isfinite(d.density_kg_m3) && d.density_kg_m3 > 0.0f)) return fail("media.density_kg_m3 must be > 0");
  if (!in_range(d.restitution_ball_ball, 0.0f, 1.0f)) return fail("media.restitution_ball_ball must be in [0, 1]");
  if (!in_range(d.restitution_ball_wall, 0.0f, 1.0f)) return fail("media.restitution_ball_wall must be in [0, 1]");
  const std::pair<const char*, float> mus[] = {
      {"friction_ball_ball", d.friction_ball_ball}, {"friction_ball_wall", d.friction_ball_wall},
      {"friction_ball_ball_static", d.friction_ball_ball_static},
      {"friction_ball_wall_static", d.friction_ball_wall_static}, {"rolling_friction", d.rolling_friction}};
  for (auto& q : mus)
    if (!(q.second >= 0.0f && std::isfinite(q.second))) return fail(std::string("media.") + q.first + " must be >= 0");
  if (d.friction_ball_ball_static < d.friction_ball_ball)
    return fail("media.friction_ball_ball_static must be >= media.friction_ball_ball");
  if (d.friction_ball_wall_static < d.friction_ball_wall)
    return fail("media.friction_ball_wall_static must be >= media.friction_ball_wall");
  if (!(d.friction_velocity_scale_m_s > 0.0f && std::isfinite(d.friction_velocity_scale_m_s)))
    return fail("media.friction_velocity_scale_m_s must be > 0");
  const SlurryParams& s = p.slurry;
  if (!in_range(s.fill_fraction, 0.0f, 0.9f)) return fail("slurry.fill_fraction must be in [0, 0.9]");
  if (!(std::isfinite(s.density_kg_m3) && s.density_kg_m3 > 0.0f)) return fail("slurry.density_kg_m3 must be > 0");
  if (!(s.viscosity_pa_s >= 0.0f && std::isfinite(s.viscosity_pa_s))) return fail("slurry.viscosity_pa_s must be >= 0");
  if (!(s.yield_stress_pa >= 0.0f && std::isfinite(s.yield_stress_pa))) return fail("slurry.yield_stress_pa must be >= 0");
  if (!(s.surface_tension_n_m >= 0.0f && std::isfinite(s.surface_tension_n_m))) return fail("slurry.surface_tension_n_m must be >= 0");
  if (!in_range(s.wall_no_slip, 0.0f, 1.0f)) return fail("slurry.wall_no_slip must be in [0, 1]");
  if (!in_range(s.ball_no_slip, 0.0f, 1.0f)) return fail("slurry.ball_no_slip must be in [0, 1]");
  if (!in_range(s.wettability, 0.0f, 1.0f)) return fail("slurry.wettability must be in [0, 1]");
  if (s.rheology > 1 || s.dye_pattern > 2) return fail("slurry enum out of range");
  const LiftersParams& l = p.lifters;
  if (l.count > 0) {
    if (!(l.height_m > 0.0f && std::isfinite(l.height_m))) return fail("lifters.height_m must be > 0");
    if (!(l.base_width_m > 0.0f && std::isfinite(l.base_width_m))) return fail("lifters.base_width_m must be > 0");
    if (!(l.top_width_m >= 0.0f && std::isfinite(l.top_width_m))) return fail("lifters.top_width_m must be >= 0");
  }
  const SimulationParams& q = p.simulation;
  if (!(q.resolution >= 4 && q.resolution <= 200)) return fail("simulation.resolution must be in [4, 200]");
  if (!(q.substeps >= 1 && q.substeps <= 64)) return fail("simulation.substeps must be in [1, 64]");
  if (!(q.pbf_iterations >= 1 && q.pbf_iterations <= 20)) return fail("simulation.pbf_iterations must be in [1, 20]");
  if (!(q.dem_iterations >= 1 && q.dem_iterations <= 20)) return fail("simulation.dem_iterations must be in [1, 20]");
  if (!(q.time_scale > 0.0f && std::isfinite(q.time_scale))) return fail("simulation.time_scale must be > 0");
  if (!(q.frame_budget_ms > 0.0f && std::isfinite(q.frame_budget_ms))) return fail("simulation.frame_budget_ms must be > 0");
  if (!(q.max_balls >= 10 && q.max_balls <= 50000)) return fail("simulation.max_balls must be in [10, 50000]");
  if (!(q.coarse_graining_k >= 1.0f && q.coarse_graining_k <= 1000.0f)) return fail("simulation.coarse_graining_k must be in [1, 1000]");
  if (q.coarse_graining_mode > 2) return fail("simulation enum out of range");
  return true;
}

// params.rs:80-113
float critical_speed_rpm(const MillParams& m) { return 42.3f / std::sqrt(m.diameter_m); }
float mill_rpm(const MillParams& m) {
  return m.speed_mode == SPEED_RPM ? m.speed_value : critical_speed_rpm(m) * m.speed_value / 100.0f;
}
float mill_percent_critical(const MillParams& m) {
  return m.speed_mode == SPEED_PERCENT_CRITICAL ? m.speed_value : 100.0f * m.speed_value / critical_speed_rpm(m);
}
float mill_omega(const MillParams& m) {
  float w = mill_rpm(m) * 2.0f * PI_F / 60.0f;
  return m.direction == DIR_CCW ? w : -w;
}

// params.rs:558-566
float true_ball_count(const Params& p) {
  float r_true = p.media.ball_diameter_m * 0.5f;
  if (r_true <= 0.0f) return 0.0f;
  float rr = mill_radius(p.mill);
  float drum_area = PI_F * (rr * rr);
  return (p.media.fill_fraction * p.media.packing_fraction_2d * drum_area) / (PI_F * r_true * r_true);
}

// params.rs:584-620
EffectiveMedia effective_media(const Params& p) {
  float true_d = p.media.ball_diameter_m;
  float rho = p.media.density_kg_m3;
  float n_true = true_ball_count(p);
  float max_balls = (float)p.simulation.max_balls;
  float k = 1.0f;
  if (p.simulation.coarse_graining_mode == CG_MANUAL) {
    k = fmax_r(p.simulation.coarse_graining_k, 1.0f);
  } else if (p.simulation.coarse_graining_mode == CG_AUTO) {
    k = (n_true > max_balls && max_balls > 0.0f) ? std::sqrt(n_true / max_balls) : 1.0f;
  }
  if (k > 1.0f) {
    uint32_t count = f2u_sat(fmax_r(std::round(n_true / (k * k)), 1.0f));
    return {true_d, true_d * k, rho, count, k};
  }
  return {true_d, true_d, rho, f2u_sat(fmax_r(std::round(n_true), 0.0f)), 1.0f};
}

// params.rs:650-658
uint32_t effective_fluid_resolution(const Params& p) {
  float radius = mill_radius(p.mill);
  float d_eff = effective_media(p).diameter_m;
  if (!(radius > 0.0f && d_eff > 0.0f)) return p.simulation.resolution;
  uint32_t min_res = f2u_sat(std::ceil(radius / d_eff));
  return std::min(std::max(p.simulation.resolution, min_res), 200u);
}

// params.rs:705-726
uint32_t effective_substeps(const Params& p) {
  float d_eff = effective_media(p).diameter_m;
  float diameter = p.mill.diameter_m;
  if (!(d_eff > 0.0f && diameter > 0.0f)) return p.simulation.substeps;
  float density_factor = clamp_r(1.0f + 2.5f * (p.media.fill_fraction - 0.30f), 1.0f, 2.0f);
  float v_ref = std::sqrt(2.0f * 9.81f * diameter);
  uint32_t min_sub = f2u_sat(fmax_r(std::ceil(v_ref * density_factor / (60.0f * 0.5f * d_eff)), 1.0f));
  uint32_t cap = f2u_sat(std::ceil(16.0f * density_factor));
  return std::max(p.simulation.substeps, std::min(min_sub, cap));
}

// web/src/params/presets.ts:91-123 (quality presets: max_balls, resolution, and the optional
// sub-step / ball-iteration / coarse-graining overrides of the impact-statistics tier)
bool preset_apply(Params* p, const char* id) {
  std::string s(id ? id : "");
  if (s == "realtime") { p->simulation.max_balls = 300; p->simulation.resolution = 25; return true; }
  if (s == "balanced") { p->simulation.max_balls = 300; p->simulation.resolution = 30; return true; }
  if (s == "accuracy") { p->simulation.max_balls = 600; p->simulation.resolution = 50; return true; }
  if (s == "impact_stats") {
    p->simulation.max_balls = 600;
    p->simulation.resolution = 25;
    p->simulation.substeps = 32;
    p->simulation.dem_iterations = 12;
    p->simulation.coarse_graining_mode = CG_OFF;
    return true;
  }
  return false;
}

// ------------------------------------------------------------------ dem.rs:230-239, 355-409
Real ball_mass(Real d, Real rho) { Real r = d * Real(0.5); return rho * PI_F * r * r; }
Real ball_inertia(Real m, Real r) { return Real(0.5) * m * r * r; }

void balls_seed_lattice(Balls* b, const EffectiveMedia& e, Real drum_r, uint64_t seed) {
  Real r = e.diameter_m * Real(0.5);
  Real mass = ball_mass(e.diameter_m, e.density_kg_m3);
  Real inertia = ball_inertia(mass, r);
  size_t count = e.ball_count;
  Rng rng(seed);
  std::vector<Vec2> x;
  if (r > Real(0.0) && count > 0) {
    Real spacing = Real(2.0) * r * Real(1.02);
    Real row_h = spacing * (std::sqrt(Real(3.0)) * Real(0.5));
    Real fill_r = fmax_r(drum_r - r, Real(0.0));
    int32_t n_rows = f2i_sat(std::ceil(Real(2.0) * fill_r / row_h)) + 1;
    bool done = false;
    for (int32_t row = -n_rows / 2; row <= n_rows / 2 && !done; ++row) {
      Real y = (Real)row * row_h;
      if (std::fabs(y) > fill_r) continue;
      Real half_width = std::sqrt(fmax_r(fill_r * fill_r - y * y, Real(0.0)));
      Real offset = (((row % 2) + 2) % 2 == 0) ? Real(0.0) : spacing * Real(0.5);
      int32_t n_cols = f2i_sat(std::floor(Real(2.0) * half_width / spacing));
      for (int32_t col = -n_cols / 2; col <= n_cols / 2; ++col) {
        Real cx = (Real)col * spacing + offset;
        if (cx * cx + y * y > fill_r * fill_r) continue;
        Real jx = rng.range_f32(-Real(0.05), Real(0.05));
        Real jy = rng.range_f32(-Real(0.05), Real(0.05));
        Vec2 jitter = Vec2(jx, jy) * r;
        x.push_back(Vec2(cx, y) + jitter);
        if (x.size() >= count) { done = true; break; }
      }
    }
  }
  if (x.size() > count) x.resize(count);
  size_t n = x.size();
  b->x = x;
  b->v.assign(n, Vec2());
  b->theta.assign(n, Real(0.0));
  b->omega.assign(n, Real(0.0));
  b->radius = r;
  b->mass = mass;
  b->inertia = inertia;
  b->true_radius = e.true_diameter_m * Real(0.5);
}

// pbf.rs:2370-2388
static Real dye_value(uint32_t pattern, Vec2 p) {
  if (pattern == DYE_LEFT_RIGHT) return p.x < Real(0.0) ? Real(0.0) : Real(1.0);
  if (pattern == DYE_TOP_BOTTOM) return p.y < Real(0.0) ? Real(0.0) : Real(1.0);
  return Real(0.0);
}

// pbf.rs:1044-1119
void fluid_seed_lattice(Fluid* f, const SlurryParams& s, Real drum_r, uint32_t res,
                        const std::vector<Vec2>& balls, Real ball_r) {
  Real dx = drum_r / (Real)std::max(res, 1u);
  Real h = Real(2.0) * dx;
  Real rest_density = s.density_kg_m3;
  Real row_h = dx * (std::sqrt(Real(3.0)) * Real(0.5));
  Real cell_area = dx * row_h;
  Real particle_mass = rest_density * cell_area;
  Real target_area = s.fill_fraction * PI_F * drum_r * drum_r;
  size_t target_count = f2u_sat(fmax_r(std::round(target_area / cell_area), Real(0.0)));
  std::vector<Vec2> x;
  std::vector<Real> dye;
  if (target_count > 0 && dx > Real(0.0)) {
    int32_t n_rows = f2i_sat(std::ceil(Real(2.0) * drum_r / row_h)) + 1;
    bool done = false;
    for (int32_t row = -n_rows / 2; row <= n_rows / 2 && !done; ++row) {
      Real y = (Real)row * row_h;
      if (std::fabs(y) > drum_r) continue;
      Real half_width = std::sqrt(fmax_r(drum_r * drum_r - y * y, Real(0.0)));
      Real offset = (((row % 2) + 2) % 2 == 0) ? Real(0.0) : dx * Real(0.5);
      int32_t n_cols = f2i_sat(std::floor(Real(2.0) * half_width / dx));
      for (int32_t col = -n_cols / 2; col <= n_cols / 2; ++col) {
        Real cx = (Real)col * dx + offset;
        if (cx * cx + y * y > drum_r * drum_r) continue;
        Vec2 p(cx, y);
        bool overlaps = false;
        for (const Vec2& b : balls)
          if ((p - b).length() < ball_r) { overlaps = true; break; }
        if (overlaps) continue;
        dye.push_back(dye_value(s.dye_pattern, p));
        x.push_back(p);
        if (x.size() >= target_count) { done = true; break; }
      }
    }
  }
  size_t n = x.size();
  f->x = x;
  f->v.assign(n, Vec2());
  f->dye = dye;
  f->viscous_guess.clear();
  f->particle_mass = particle_mass;
  f->h = h;
  f->rest_density = rest_density;
}

// ------------------------------------------------------------------ grid.rs:101-270
UniformGrid UniformGrid::build(const std::vector<Vec2>& pts, Real cell) {
  UniformGrid g;
  g.cell_size = cell;
  std::vector<std::pair<std::pair<int32_t, int32_t>, uint32_t>> keyed;
  keyed.reserve(pts.size());
  int32_t min_cx = INT32_MAX, min_cy = INT32_MAX, max_cx = INT32_MIN, max_cy = INT32_MIN;
  for (size_t i = 0; i < pts.size(); ++i) {
    if (!pts[i].is_finite()) continue;
    auto k = cell_key(pts[i], cell);
    min_cx = std::min(min_cx, k.first);
    min_cy = std::min(min_cy, k.second);
    max_cx = std::max(max_cx, k.first);
    max_cy = std::max(max_cy, k.second);
    keyed.push_back({k, (uint32_t)i});
  }
  if (keyed.empty()) {
    g.dense = false;
    g.cell_start.assign(1, 0);
    return g;
  }
  int64_t width = (int64_t)max_cx - (int64_t)min_cx + 1;
  int64_t height = (int64_t)max_cy - (int64_t)min_cy + 1;
  unsigned __int128 total = (unsigned __int128)(uint64_t)width * (uint64_t)height;
  uint64_t budget = 2ull * (uint64_t)keyed.size() + 512ull;
  if (total <= budget) {
    g.dense = true;
    g.min_cx = min_cx;
    g.min_cy = min_cy;
    g.width = width;
    g.height = height;
    size_t cells = (size_t)(width * height);
    g.cell_start.assign(cells + 1, 0);
    auto didx = [&](std::pair<int32_t, int32_t> k) {
      return (size_t)(((int64_t)k.first - min_cx) * height + ((int64_t)k.second - min_cy));
    };
    for (auto& kv : keyed) g.cell_start[didx(kv.first) + 1] += 1;
    for (size_t i = 1; i < g.cell_start.size(); ++i) g.cell_start[i] += g.cell_start[i - 1];
    std::vector<uint32_t> cursor = g.cell_start;
    g.indices.assign(keyed.size(), 0);
    for (auto& kv : keyed) {
      size_t k = didx(kv.first);
      g.indices[cursor[k]] = kv.second;
      cursor[k] += 1;
    }
  } else {
    g.dense = false;
    std::stable_sort(keyed.begin(), keyed.end(),
                     [](const std::pair<std::pair<int32_t, int32_t>, uint32_t>& a,
                        const std::pair<std::pair<int32_t, int32_t>, uint32_t>& b) { return a.first < b.first; });
    g.cell_start.assign(1, 0);
    size_t i = 0;
    while (i < keyed.size()) {
      auto key = keyed[i].first;
      size_t j = i;
      while (j < keyed.size() && keyed[j].first == key) { g.indices.push_back(keyed[j].second); ++j; }
      g.keys.push_back(key);
      g.cell_start.push_back((uint32_t)j);
      i = j;
    }
  }
  return g;
}

bool UniformGrid::cell_range(std::pair<int32_t, int32_t> key, size_t* s, size_t* e) const {
  if (dense) {
    int64_t dcx = (int64_t)key.first - (int64_t)min_cx;
    int64_t dcy = (int64_t)key.second - (int64_t)min_cy;
    if (dcx < 0 || dcy < 0 || dcx >= width || dcy >= height) return false;
    size_t k = (size_t)(dcx * height + dcy);
    *s = cell_start[k];
    *e = cell_start[k + 1];
    return *s != *e;
  }
  auto it = std::lower_bound(keys.begin(), keys.end(), key);
  if (it == keys.end() || *it != key) return false;
  size_t idx = (size_t)(it - keys.begin());
  *s = cell_start[idx];
  *e = cell_start[idx + 1];
  return true;
}

std::vector<std::pair<uint32_t, uint32_t>> candidate_pairs(const std::vector<Vec2>& pts, Real cell) {
  std::vector<std::pair<uint32_t, uint32_t>> out;
  UniformGrid g = UniformGrid::build(pts, cell);
  g.for_each_candidate_pair([&](uint32_t i, uint32_t j) { out.push_back({i, j}); });
  return out;
}

// ------------------------------------------------------------------ geometry.rs
Real Drum::sdf(Vec2 p) const {
  Real d = radius_m - p.length();
  if (lifters.count == 0) return d;
  return fmin_r(d, sdf_lifters(p));
}

Real Drum::sdf_lifters(Vec2 p) const {
  uint32_t n = lifters.count;
  const Real rads_per_deg = PI_F / Real(180.0);
  Real phase = lifters.phase_deg * rads_per_deg;
  Real max_inside = -INFINITY;
  for (uint32_t k = 0; k < n; ++k) {
    Real theta_i = phase + (Real)k * TAU_F / (Real)n;
    Real s = sinf_r(theta_i), c = cosf_r(theta_i);
    Real pr = p.x * c + p.y * s;
    Real pt = -p.x * s + p.y * c;
    Real inside = lifter_cross_section_sdf(pr, pt, radius_m, lifters.height_m, lifters.base_width_m * Real(0.5),
                                            lifters.top_width_m * Real(0.5));
    max_inside = fmax_r(max_inside, inside);
  }
  return -max_inside;
}

void Drum::sdf_world(Vec2 pw, Real angle, Real* d, Vec2* normal) const {
  if (!pw.is_finite()) { *d = Real(0.0); *normal = Vec2(); return; }
  Vec2 to_local = Vec2::from_angle(-angle);
  Vec2 pl = rotate(pw, to_local);
  const Real EPS = Real(1e-4);
  Real dd = sdf(pl);
  Real gx = sdf(pl + Vec2(EPS, Real(0.0))) - sdf(pl - Vec2(EPS, Real(0.0)));
  Real gy = sdf(pl + Vec2(Real(0.0), EPS)) - sdf(pl - Vec2(Real(0.0), EPS));
  Vec2 grad = Vec2(gx, gy) / (Real(2.0) * EPS);
  Vec2 nl = grad.length_squared() > Real(1e-12) ? grad.normalize() : -pl.normalize_or_zero();
  Vec2 to_world = Vec2::from_angle(angle);
  *d = dd;
  *normal = rotate(nl, to_world);
}

bool Drum::toi_swept(Vec2 x0, Vec2 x1, Real a0, Real a1, Real radius, Real* t_out) const {
  Vec2 local0 = rotate(x0, Vec2::from_angle(-a0));
  if (sdf(local0) - radius <= Real(0.0)) return false;
  Vec2 path = x1 - x0;
  Real path_len = path.length();
  Real dangle = a1 - a0;
  Real pos_bound = x0.length() + path_len;
  Real bound = path_len + std::fabs(dangle) * pos_bound;
  if (bound < Real(1e-9)) return false;
  Real t = Real(0.0);
  for (int it = 0; it < 32; ++it) {
    Real angle_t = a0 + dangle * t;
    Vec2 x_t = x0 + path * t;
    Vec2 local = rotate(x_t, Vec2::from_angle(-angle_t));
    Real d = sdf(local) - radius;
    if (d <= Real(0.0)) { *t_out = t; return true; }
    Real step_t = fmax_r(d / bound, Real(1e-6));
    t += step_t;
    if (t >= Real(1.0)) return false;
  }
  *t_out = fmin_r(t, Real(1.0));
  return true;
}

Real lifter_cross_section_sdf(Real pr, Real pt, Real r, Real height, Real base_half, Real top_half) {
  Real r_top = r - height;
  Vec2 verts[4] = {Vec2(r, -base_half), Vec2(r, base_half), Vec2(r_top, top_half), Vec2(r_top, -top_half)};
  return convex_polygon_sdf(Vec2(pr, pt), verts, 4);
}

Real convex_polygon_sdf(Vec2 p, const Vec2* verts, int n) {
  Real min_dist_sq = Real(3.40282347e38);
  bool inside = true;
  for (int i = 0; i < n; ++i) {
    Vec2 a = verts[i];
    Vec2 b = verts[(i + 1) % n];
    Vec2 edge = b - a;
    Vec2 to_p = p - a;
    Real len_sq = edge.length_squared();
    if (len_sq < Real(1e-12)) continue;
    Real t = clamp_r(to_p.dot(edge) / len_sq, Real(0.0), Real(1.0));
    Vec2 closest = a + edge * t;
    min_dist_sq = fmin_r(min_dist_sq, (p - closest).length_squared());
    Real cross = edge.x * to_p.y - edge.y * to_p.x;
    if (cross < Real(0.0)) inside = false;
  }
  Real dist = std::sqrt(min_dist_sq);
  return inside ? dist : -dist;
}

}  // namespace orc
