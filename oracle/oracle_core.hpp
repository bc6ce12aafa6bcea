// Oracle: CPU restatement of MillDynamics3's per-sub-step hot path (Rust, crates/mill-core).
//
// TEST INFRASTRUCTURE ONLY. Nothing in the shipped library links, loads or calls this code; only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only as the checker
// or the timed CPU reference.
//
// Arithmetic follows the reference in f32 with IEEE division and square root and no fused
// multiply-add (build with -ffp-contract=off, no fast-math), and in the same evaluation order as
// the Rust source (left to right; Rust never reassociates or contracts). glam 0.29's Vec2 is
// restated here with the semantics the reference relies on: dot = x*x' + y*y', length =
// sqrt(dot), normalize = v * (1 / length), Vec2 / s divides each component.
//
// Parity status. The reference ships no golden state vectors, and its toolchain (cargo/rustc) is
// absent, so bit-level parity of this restatement against the Rust build is unpinned. It is pinned
// instead against the reference's own unit-test assertions for this path (ported under tests/).
// Transcendentals are the one known source of platform drift: the reference computes
// Vec2::from_angle through the libm crate (a musl port) and f32 exp/atan2/powf/log10/sin/cos
// through the platform libm; this restatement calls glibc for all of them.
#pragma once

#include <cmath>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

struct MgMetrics;  // include/millgpu.h

namespace orc {

// The arithmetic type of the restated kernels. The parity oracle is built with Real = float (the
// reference's f32); the FP64 oracle is the same source built with -DORC_REAL=double, for the
// per-output error reports of the f32 path. Params and their derived quantities stay f32 in both
// builds (they are the reference's f32 inputs), so both builds step the same inputs.
#ifndef ORC_REAL
#define ORC_REAL float
#endif
using Real = ORC_REAL;

constexpr Real PI_F = Real(3.14159265358979323846);
constexpr Real TAU_F = Real(6.28318530717958647692);

// Transcendentals. Every f32 exp/sin/cos/atan2/log10 of the reference is evaluated here as the
// f32 rounding of the f64 function (error <= 0.5 ulp + 2^-29, against <= ~0.502 ulp for the
// platform's f32 functions the Rust build calls), so that the device path, which evaluates them
// the same way, can agree bit for bit. With T = double they are the f64 functions themselves.
template <class T> inline T expf_r(T x) { return (T)std::exp((double)x); }
template <class T> inline T sinf_r(T x) { return (T)std::sin((double)x); }
template <class T> inline T cosf_r(T x) { return (T)std::cos((double)x); }
template <class T> inline T atan2f_r(T y, T x) { return (T)std::atan2((double)y, (double)x); }
template <class T> inline T log10f_r(T x) { return (T)std::log10((double)x); }

// f32::max / f32::min (IEEE maxNum/minNum: a NaN operand yields the other operand).
template <class T> inline T fmax_r(T a, T b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a > b ? a : b;
}
template <class T> inline T fmin_r(T a, T b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a < b ? a : b;
}
inline double dmax_r(double a, double b) { return fmax_r<double>(a, b); }
// f32::clamp: `if x < lo {lo}; if x > hi {hi}` (a NaN passes through).
template <class T> inline T clamp_r(T x, T lo, T hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
inline double dclamp_r(double x, double lo, double hi) { return clamp_r<double>(x, lo, hi); }
// Rust `f as i32`: saturating, NaN -> 0.
template <class T> inline int32_t f2i_sat(T f) {
  if (std::isnan(f)) return 0;
  if (f >= T(2147483648.0)) return INT32_MAX;
  if (f <= -T(2147483648.0)) return INT32_MIN;
  return (int32_t)f;
}
// Rust `f as u32` / `f as usize`: saturating at 0 below, NaN -> 0.
template <class T> inline uint32_t f2u_sat(T f) {
  if (std::isnan(f) || f <= T(0.0)) return 0;
  if (f >= T(4294967296.0)) return UINT32_MAX;
  return (uint32_t)f;
}
inline uint64_t d2u64_sat(double f) {
  if (std::isnan(f) || f <= 0.0) return 0;
  if (f >= 18446744073709551616.0) return UINT64_MAX;
  return (uint64_t)f;
}
inline int32_t sat_add_i32(int32_t a, int32_t b) {
  int64_t s = (int64_t)a + (int64_t)b;
  if (s > INT32_MAX) return INT32_MAX;
  if (s < INT32_MIN) return INT32_MIN;
  return (int32_t)s;
}
template <class T> inline T signum_r(T x) {
  if (std::isnan(x)) return x;
  return std::signbit(x) ? -T(1.0) : T(1.0);
}
// f32::rem_euclid: r = self % rhs; if r < 0 { r + |rhs| } else { r }.
template <class T> inline T rem_euclid_r(T x, T m) {
  T r = std::fmod(x, m);
  return r < T(0.0) ? r + std::fabs(m) : r;
}
// powi lowered by LLVM to binary exponentiation (x^3 = x * x^2, x^5 = x * x^4, x^6 = x^2 * x^4,
// x^8 = x^4 * x^4); the same products compiler-rt's __powisf2 forms.
template <class T> inline T powi3(T x) { return x * (x * x); }
template <class T> inline T powi5(T x) { T x2 = x * x; T x4 = x2 * x2; return x * x4; }
template <class T> inline T powi6(T x) { T x2 = x * x; T x4 = x2 * x2; return x2 * x4; }
template <class T> inline T powi8(T x) { T x2 = x * x; T x4 = x2 * x2; return x4 * x4; }

struct Vec2 {
  Real x, y;
  Vec2() : x(Real(0.0)), y(Real(0.0)) {}
  Vec2(Real a, Real b) : x(a), y(b) {}
  Vec2 operator+(Vec2 o) const { return Vec2(x + o.x, y + o.y); }
  Vec2 operator-(Vec2 o) const { return Vec2(x - o.x, y - o.y); }
  Vec2 operator-() const { return Vec2(-x, -y); }
  Vec2 operator*(Real s) const { return Vec2(x * s, y * s); }
  Vec2 operator/(Real s) const { return Vec2(x / s, y / s); }
  Vec2& operator+=(Vec2 o) { x += o.x; y += o.y; return *this; }
  Vec2& operator-=(Vec2 o) { x -= o.x; y -= o.y; return *this; }
  Vec2& operator*=(Real s) { x *= s; y *= s; return *this; }
  Real dot(Vec2 o) const { return (x * o.x) + (y * o.y); }
  Real length_squared() const { return dot(*this); }
  Real length() const { return std::sqrt(dot(*this)); }
  bool is_finite() const { return std::isfinite(x) && std::isfinite(y); }
  Vec2 normalize() const { Real rcp = Real(1.0) / length(); return *this * rcp; }
  Vec2 normalize_or_zero() const {
    Real rcp = Real(1.0) / length();
    if (std::isfinite(rcp) && rcp > Real(0.0)) return *this * rcp;
    return Vec2();
  }
  static Vec2 from_angle(Real a) { return Vec2(cosf_r(a), sinf_r(a)); }
};
inline Vec2 operator*(Real s, Vec2 v) { return Vec2(s * v.x, s * v.y); }
inline Real cross2(Vec2 a, Vec2 b) { return a.x * b.y - a.y * b.x; }

// ---------------------------------------------------------------- params (params.rs)

enum SpeedMode : uint32_t { SPEED_RPM = 0, SPEED_PERCENT_CRITICAL = 1 };
enum Direction : uint32_t { DIR_CCW = 0, DIR_CW = 1 };
enum CoarseMode : uint32_t { CG_AUTO = 0, CG_OFF = 1, CG_MANUAL = 2 };
enum Rheology : uint32_t { RHEO_NEWTONIAN = 0, RHEO_BINGHAM = 1 };
enum DyePattern : uint32_t { DYE_LEFT_RIGHT = 0, DYE_TOP_BOTTOM = 1, DYE_NONE = 2 };

struct MillParams { float diameter_m; uint32_t speed_mode; float speed_value; uint32_t direction; };
struct MediaParams {
  float ball_diameter_m, fill_fraction, packing_fraction_2d, density_kg_m3;
  float restitution_ball_ball, restitution_ball_wall, friction_ball_ball, friction_ball_wall;
  float friction_ball_ball_static, friction_ball_wall_static, friction_velocity_scale_m_s;
  float rolling_friction;
};
struct SlurryParams {
  uint32_t enabled;
  float fill_fraction, density_kg_m3, viscosity_pa_s;
  uint32_t rheology;
  float yield_stress_pa, wall_no_slip, ball_no_slip, wettability, surface_tension_n_m;
  uint32_t dye_pattern;
};
struct LiftersParams { uint32_t count; float height_m, base_width_m, top_width_m, phase_deg; };
struct SimulationParams {
  uint32_t resolution, substeps, pbf_iterations, dem_iterations;
  float time_scale, frame_budget_ms;
  uint32_t max_balls, pad0;
  uint64_t seed;
  uint32_t coarse_graining_mode;
  float coarse_graining_k;
};
struct Params {
  MillParams mill;
  MediaParams media;
  SlurryParams slurry;
  LiftersParams lifters;
  SimulationParams simulation;
};
struct EffectiveMedia { float true_diameter_m, diameter_m, density_kg_m3; uint32_t ball_count; float scale_factor; };

Params params_default();
bool params_validate(const Params& p, std::string* err);
float critical_speed_rpm(const MillParams& m);
float mill_rpm(const MillParams& m);
float mill_percent_critical(const MillParams& m);
float mill_omega(const MillParams& m);
inline float mill_radius(const MillParams& m) { return m.diameter_m * 0.5f; }
float true_ball_count(const Params& p);
EffectiveMedia effective_media(const Params& p);
uint32_t effective_fluid_resolution(const Params& p);
uint32_t effective_substeps(const Params& p);
bool preset_apply(Params* p, const char* id);

// ---------------------------------------------------------------- rng.rs
struct Rng {
  uint64_t state;
  explicit Rng(uint64_t seed) : state(seed == 0 ? 0x9E3779B97F4A7C15ull : seed) {}
  uint64_t next_u64() {
    uint64_t x = state;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    state = x;
    return x * 0x2545F4914F6CDD1Dull;
  }
  float next_f32() { return (float)(next_u64() >> 40) / (float)(1u << 24); }
  float range_f32(float lo, float hi) { return lo + next_f32() * (hi - lo); }
};

// ---------------------------------------------------------------- grid.rs
struct UniformGrid {
  Real cell_size = Real(1.0);
  bool dense = false;
  int32_t min_cx = 0, min_cy = 0;
  int64_t width = 0, height = 0;
  std::vector<std::pair<int32_t, int32_t>> keys;  // sparse layout only
  std::vector<uint32_t> cell_start;
  std::vector<uint32_t> indices;

  static std::pair<int32_t, int32_t> cell_key(Vec2 p, Real cell) {
    return {f2i_sat(std::floor(p.x / cell)), f2i_sat(std::floor(p.y / cell))};
  }
  static UniformGrid build(const std::vector<Vec2>& pts, Real cell);
  bool cell_range(std::pair<int32_t, int32_t> key, size_t* s, size_t* e) const;
  template <class F> void for_each_candidate_pair(F f) const;
  template <class F> void for_each_near(Vec2 p, F f) const;
};

template <class F>
void UniformGrid::for_each_candidate_pair(F f) const {
  static const int32_t FWD[4][2] = {{1, 0}, {1, 1}, {0, 1}, {-1, 1}};
  auto visit_cell = [&](int32_t cx, int32_t cy, size_t s, size_t e) {
    for (size_t a = s; a < e; ++a)
      for (size_t b = a + 1; b < e; ++b) {
        uint32_t i = indices[a], j = indices[b];
        f(i < j ? i : j, i < j ? j : i);
      }
    for (int q = 0; q < 4; ++q) {
      std::pair<int32_t, int32_t> key = {sat_add_i32(cx, FWD[q][0]), sat_add_i32(cy, FWD[q][1])};
      if (key.first == cx && key.second == cy) continue;
      size_t os, oe;
      if (!cell_range(key, &os, &oe)) continue;
      for (size_t a = s; a < e; ++a)
        for (size_t b = os; b < oe; ++b) {
          uint32_t i = indices[a], j = indices[b];
          f(i < j ? i : j, i < j ? j : i);
        }
    }
  };
  if (dense) {
    size_t total = (size_t)(width * height);
    for (size_t k = 0; k < total; ++k) {
      size_t s = cell_start[k], e = cell_start[k + 1];
      if (s == e) continue;
      int32_t cx = min_cx + (int32_t)((int64_t)k / height);
      int32_t cy = min_cy + (int32_t)((int64_t)k % height);
      visit_cell(cx, cy, s, e);
    }
  } else {
    for (size_t idx = 0; idx < keys.size(); ++idx)
      visit_cell(keys[idx].first, keys[idx].second, cell_start[idx], cell_start[idx + 1]);
  }
}

template <class F>
void UniformGrid::for_each_near(Vec2 p, F f) const {
  if (!p.is_finite()) return;
  auto c = cell_key(p, cell_size);
  std::pair<int32_t, int32_t> ks[9];
  int nk = 0;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      std::pair<int32_t, int32_t> key = {sat_add_i32(c.first, dx), sat_add_i32(c.second, dy)};
      bool seen = false;
      for (int q = 0; q < nk; ++q) seen = seen || (ks[q] == key);
      if (!seen) ks[nk++] = key;
    }
  for (int q = 0; q < nk; ++q) {
    size_t s, e;
    if (!cell_range(ks[q], &s, &e)) continue;
    for (size_t a = s; a < e; ++a) f(indices[a]);
  }
}

// ---------------------------------------------------------------- geometry.rs
struct Drum {
  Real radius_m = Real(0.0);
  Real omega = Real(0.0);
  LiftersParams lifters{};
  Real sdf(Vec2 p_local) const;
  Real sdf_lifters(Vec2 p_local) const;
  void sdf_world(Vec2 p_world, Real drum_angle, Real* d, Vec2* normal) const;
  Vec2 wall_velocity(Vec2 p) const { return omega * Vec2(-p.y, p.x); }
  bool toi_swept(Vec2 x0, Vec2 x1, Real a0, Real a1, Real radius, Real* t_out) const;
};
inline Vec2 rotate(Vec2 v, Vec2 u) { return Vec2(v.x * u.x - v.y * u.y, v.x * u.y + v.y * u.x); }
Real convex_polygon_sdf(Vec2 p, const Vec2* verts, int n);
Real lifter_cross_section_sdf(Real pr, Real pt, Real r, Real height, Real base_half, Real top_half);

// ---------------------------------------------------------------- dem.rs / pbf.rs state
struct Balls {
  std::vector<Vec2> x, v;
  std::vector<Real> theta, omega;
  Real radius = Real(0.0), mass = Real(0.0), inertia = Real(0.0), true_radius = Real(0.0);
  size_t len() const { return x.size(); }
};
struct Fluid {
  std::vector<Vec2> x, v;
  std::vector<Real> dye;
  std::vector<Vec2> viscous_guess;
  Real particle_mass = Real(0.0), h = Real(0.0), rest_density = Real(0.0);
  size_t len() const { return x.size(); }
};

constexpr int WALL_IMPULSE_BINS = 32;
constexpr int IMPACT_BINS = 12;
constexpr uint32_t WALL_ID = 0xFFFFFFFFu;

struct CouplingImpulses {
  std::vector<Vec2> impulses;
  std::vector<Real> angular_impulses;
  uint32_t clamp_hits = 0;
  Vec2 fluid_momentum_change;
  void zeros(size_t nb) {
    impulses.assign(nb, Vec2());
    angular_impulses.assign(nb, Real(0.0));
    clamp_hits = 0;
    fluid_momentum_change = Vec2();
  }
};
struct FluidStepStats {
  uint32_t viscosity_iterations = 0;
  Real mean_shear_rate_per_s = Real(0.0);
  uint32_t coupling_clamp_hits = 0;
  Real wall_work_j = Real(0.0);
  Real wall_impulse[2] = {Real(0.0), Real(0.0)};
  Real wall_angular_impulse = Real(0.0);
  Real wall_normal_impulse_by_angle[WALL_IMPULSE_BINS] = {};
  Real ke_delta_noslip_j = Real(0.0), ke_delta_drag_j = Real(0.0), ke_delta_buoyancy_j = Real(0.0);
  Real ke_delta_viscosity_j = Real(0.0), ke_delta_clamp_j = Real(0.0);
};
struct DemStepStats {
  Real wall_work_j = Real(0.0);
  uint32_t collision_count = 0;
  uint32_t impact_energy_histogram[IMPACT_BINS] = {};
  Real dissipated_energy_j = Real(0.0);
  Real max_substep_displacement_over_diameter = Real(0.0);
  Real coupling_work_j = Real(0.0);
};
struct ImpactRecord {
  uint32_t kind;  // 0 ball-ball, 1 ball-wall
  uint32_t ball, partner;
  float normal_speed, slip_speed, restitution;
};
// Counters of one sub-step (stage_timing.rs Counters semantics), for diagnostics and parity.
struct StepCounters {
  uint32_t density_iters = 0, cg_iters = 0, n_groups = 0, n_links = 0, links_in_range = 0;
  uint32_t n_ball_pairs = 0, n_fluid_edges = 0, n_active_contacts = 0;
  uint32_t n_coupling_items = 0, ccd_clamps = 0;
};

// Last sub-step's internal structures, kept for parity checks of the device path.
struct Debug {
  std::vector<uint32_t> nbr_offsets, nbrs;
  std::vector<std::pair<uint32_t, uint32_t>> ball_pairs;
};

void fluid_seed_lattice(Fluid* f, const SlurryParams& s, Real drum_r, uint32_t res,
                        const std::vector<Vec2>& balls, Real ball_r);
void balls_seed_lattice(Balls* b, const EffectiveMedia& e, Real drum_r, uint64_t seed);
Real ball_mass(Real d, Real rho);
Real ball_inertia(Real m, Real r);

// Reduction mode of the viscosity solve's inner products: 0 = the reference's sequential f32 sums,
// 1 = f64 sums (the device path's FP64 mode).
struct SolveOptions { int cg_fp64 = 0; };

void fluid_step_coupled(Fluid* f, const Drum& drum, Real drum_angle, const SlurryParams& slurry,
                        uint32_t iterations, Real dt, const Balls& balls, CouplingImpulses* out,
                        FluidStepStats* stats, StepCounters* ctr, Debug* dbg, const SolveOptions& opt);
DemStepStats dem_step_recorded(Balls* b, const Drum& drum, Real drum_angle, const MediaParams& media,
                               uint32_t iterations, Real dt, const CouplingImpulses* ext,
                               std::vector<ImpactRecord>* impacts, StepCounters* ctr, Debug* dbg);
double dem_mechanical_energy_f64(const Balls& b);
double fluid_mechanical_energy(const Fluid& f);
std::vector<Real> fluid_densities(const Fluid& f);
std::vector<std::pair<uint32_t, uint32_t>> candidate_pairs(const std::vector<Vec2>& pts, Real cell);
void neighbor_lists(const std::vector<Vec2>& x, Real h, std::vector<uint32_t>* offsets,
                    std::vector<uint32_t>* nbrs);
Real effective_friction(Real mu_k, Real mu_s, Real v_t, Real vs);
int impact_energy_bin(Real e);
Real restitution_velocity_threshold(Real r);

// ---------------------------------------------------------------- stress.rs
constexpr int SE_BINS = 28;
struct StressAccum {
  double count_rate[4] = {}, se_hat_rate[4] = {}, hist_rate[SE_BINS] = {}, above_rate_j[6] = {};
  double cum_wall_j = 0.0, cum_above_j[6] = {};
  std::map<std::pair<uint32_t, uint32_t>, double> last_counted;
  bool has_debounce = false;
  double debounce_factor = 0.25;
  uint64_t updates = 0;
  void update(const std::vector<ImpactRecord>& recs, double m3, double scale_j, double d, double now_s,
              double sub_dt, double alpha, double wall_work_j);
  double total_rate() const { return count_rate[0] + count_rate[1] + count_rate[2] + count_rate[3]; }
};
int se_bin(double e_hat);

// ---------------------------------------------------------------- lib.rs
struct EnergyBudget {
  double elapsed_s = 0, shaft_work_j = 0, dem_wall_work_j = 0, fluid_wall_work_j = 0;
  double ball_contact_dissipation_j = 0, fluid_wall_slip_j = 0, fluid_viscous_j = 0;
  double fluid_clamp_removed_j = 0, interface_created_j = 0, delta_mechanical_j = 0;
  double unattributed_j = 0, fluid_wall_angular_impulse = 0;
};

struct Simulation {
  Params params{};
  Real drum_angle = Real(0.0);
  double sim_time = 0.0;
  Balls balls;
  Fluid fluid;
  FluidStepStats fluid_stats;
  Real power_draw_w = Real(0.0), torque_nm = Real(0.0), collision_rate_per_s = Real(0.0), dissipated_power_w = Real(0.0);
  std::vector<ImpactRecord> impact_log;
  StressAccum stress;
  Real max_substep_displacement_over_diameter = Real(0.0);
  uint32_t coupling_clamp_hits = 0;
  EnergyBudget energy_budget;
  double energy_budget_e0 = 0.0;
  StepCounters last_counters;
  Debug dbg;
  SolveOptions opt;
  DemStepStats last_dem_stats;

  static bool build(const Params& p, const std::vector<Vec2>* initial, Simulation* out, std::string* err);
  double total_mechanical_energy_j() const;
  EnergyBudget energy_budget_now() const;
  Real fixed_sub_dt() const;
  void reset_frame_stats();
  void step(Real dt);
  void step_fixed();
  void advance_one_sub_step(Real sub_dt);
  void update_grinding_stats(const DemStepStats& s, Real fluid_wall_work, Real sub_dt, Real omega);
  void stress_scales(double* m3, double* scale_j, double* d) const;
  Drum drum() const;
};

bool mixing_index(const Fluid& f, const Drum& d, Real* out);
void metrics_compute(const Balls& b, const Fluid& f, const Drum& d, Real drum_angle, ::MgMetrics* out);
Real surface_phi_full(const Fluid& f);
std::vector<Real> surface_build_field(const Fluid& f, const Drum& drum, Real drum_angle);
std::vector<Real> surface_extract_flat(const Fluid& f, const Drum& drum, Real drum_angle);
uint64_t state_hash(const Balls& b, const Fluid& f, bool extended);

}  // namespace orc
