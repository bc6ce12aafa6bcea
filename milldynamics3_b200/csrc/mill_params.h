// Host-side parameter logic of the library: Params defaults, validation, quality presets and the
// derived counts (params.rs, web/src/params/presets.ts), the xorshift64* RNG (rng.rs) and the two
// lattice seeders (dem.rs:355-409, pbf.rs:1044-1119). Pure f32 host arithmetic in the reference's
// order; transcendentals as the f32 rounding of the f64 libm function (the device does the same).
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/millgpu.h"

namespace mgh {

constexpr float PI_F = 3.14159265358979323846f;
constexpr float TAU_F = 6.28318530717958647692f;

inline float expf_r(float x) { return (float)std::exp((double)x); }
inline float sinf_r(float x) { return (float)std::sin((double)x); }
inline float cosf_r(float x) { return (float)std::cos((double)x); }
inline float fmax_r(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a > b ? a : b;
}
inline float fmin_r(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a < b ? a : b;
}
inline float clamp_r(float x, float lo, float hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
inline uint32_t f2u_sat(float f) {
  if (std::isnan(f) || f <= 0.0f) return 0;
  if (f >= 4294967296.0f) return UINT32_MAX;
  return (uint32_t)f;
}
inline int32_t f2i_sat(float f) {
  if (std::isnan(f)) return 0;
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (int32_t)f;
}
inline float rem_euclid_r(float x, float m) {
  float r = std::fmod(x, m);
  return r < 0.0f ? r + std::fabs(m) : r;
}

struct Effective {
  float true_diameter_m, diameter_m, density_kg_m3;
  uint32_t ball_count;
  float scale_factor;
};

MgParams params_default();
bool params_validate(const MgParams& p, std::string* err);
bool preset_apply(MgParams* p, const char* id);
float critical_speed_rpm(const MgMillParams& m);
float mill_rpm(const MgMillParams& m);
float mill_percent_critical(const MgMillParams& m);
float mill_omega(const MgMillParams& m);
inline float mill_radius(const MgMillParams& m) { return m.diameter_m * 0.5f; }
float true_ball_count(const MgParams& p);
Effective effective_media(const MgParams& p);
uint32_t effective_fluid_resolution(const MgParams& p);
uint32_t effective_substeps(const MgParams& p);

struct Balls {
  std::vector<float> x, v, theta, omega;  // x, v interleaved
  float radius = 0, mass = 0, inertia = 0, true_radius = 0;
  size_t len() const { return theta.size(); }
};
struct Fluid {
  std::vector<float> x, v, dye, guess;  // guess empty or interleaved n
  float particle_mass = 0, h = 0, rest_density = 0;
  size_t len() const { return dye.size(); }
};

void seed_balls(Balls* b, const Effective& e, float drum_r, uint64_t seed);
void seed_fluid(Fluid* f, const MgSlurryParams& s, float drum_r, uint32_t res, const std::vector<float>& balls_xy,
                float ball_r);
float ball_mass(float d, float rho);
double balls_energy_f64(const Balls& b);
double fluid_energy_f64(const Fluid& f);

}  // namespace mgh
