// Oracle (test infrastructure only): metrics::compute (metrics.rs:195-273) and the functions it
// calls (metrics.rs:281-711), restated in plain C++ over the oracle's state, for checking the
// device's metrics kernel. Each function cites the reference lines it follows.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../include/millgpu.h"
#include "oracle_core.hpp"

namespace orc {
namespace {

constexpr float WALL_MARGIN_BALL_RADII = 2.5f;                 // metrics.rs:37
constexpr size_t MIN_WALL_BALLS = 6;                           // metrics.rs:41
constexpr float CENTRIFUGE_GAP_THRESHOLD_RAD = PI_F * 0.3f;    // metrics.rs:45
constexpr float POOL_WALL_MARGIN_H = 1.5f;                     // metrics.rs:48
constexpr float POOL_DEPTH_BAND_RAD = 5.0f * PI_F / 180.0f;    // metrics.rs:51
constexpr float FRAC_PI_2_F = 1.57079632679489661923f;

float wall_distance(const Drum& d, Vec2 p, float drum_angle) {
  float dist;
  Vec2 nrm;
  d.sdf_world(p, drum_angle, &dist, &nrm);
  return dist;
}

// metrics.rs:281-284
float angular_separation(float a, float b) {
  float d = rem_euclid_r(a - b, TAU_F);
  return fmin_r(d, TAU_F - d);
}

// metrics.rs:292-307 over angles sorted ascending (n >= 2)
void largest_gap_cluster_bounds(const std::vector<float>& a, float* start, float* end, float* gap) {
  const size_t n = a.size();
  float max_gap = a[0] + TAU_F - a[n - 1];
  size_t gap_k = n - 1;
  for (size_t i = 0; i + 1 < n; ++i) {
    float g = a[i + 1] - a[i];
    if (g > max_gap) {
      max_gap = g;
      gap_k = i;
    }
  }
  *end = a[gap_k];
  *start = a[(gap_k + 1) % n];
  *gap = max_gap;
}

// sort_by(partial_cmp): a stable ascending sort (-0.0 and 0.0 compare equal)
void sort_angles(std::vector<float>* a) {
  std::stable_sort(a->begin(), a->end(), [](float x, float y) { return x < y; });
}

float world_angle(Vec2 p) { return rem_euclid_r(atan2f_r(p.y, p.x), TAU_F); }

}  // namespace

// metrics.rs:195-273 (the fields compute fills)
void metrics_compute(const Balls& b, const Fluid& f, const Drum& d, float drum_angle, MgMetrics* o) {
  std::memset(o, 0, sizeof(*o));
  const size_t nb = b.len(), nf = f.len();
  // charge_toe_shoulder, metrics.rs:327-360
  if (nb > 0) {
    const float margin = WALL_MARGIN_BALL_RADII * b.radius;
    std::vector<float> angles;
    for (size_t i = 0; i < nb; ++i)
      if (wall_distance(d, b.x[i], drum_angle) < margin) angles.push_back(world_angle(b.x[i]));
    if (angles.size() >= MIN_WALL_BALLS) {
      sort_angles(&angles);
      float cs, ce, gap;
      largest_gap_cluster_bounds(angles, &cs, &ce, &gap);
      if (!(gap <= CENTRIFUGE_GAP_THRESHOLD_RAD)) {
        o->valid |= MG_METRIC_TOE_SHOULDER;
        o->toe_angle_rad = d.omega >= 0.0f ? cs : ce;
        o->shoulder_angle_rad = d.omega >= 0.0f ? ce : cs;
      }
    }
    // charge_centroid, metrics.rs:362-369
    Vec2 sum;
    for (size_t i = 0; i < nb; ++i) sum = sum + b.x[i];
    const Vec2 c = sum / (float)nb;
    o->valid |= MG_METRIC_CENTROID;
    o->charge_centroid_m[0] = c.x;
    o->charge_centroid_m[1] = c.y;
  }
  if (nf > 0) {
    const float margin = POOL_WALL_MARGIN_H * f.h;
    // slurry_pool_angular_extent, metrics.rs:377-400
    std::vector<float> angles;
    std::vector<Vec2> pts;
    for (size_t i = 0; i < nf; ++i) {
      if (wall_distance(d, f.x[i], drum_angle) < margin) angles.push_back(world_angle(f.x[i]));
      else pts.push_back(f.x[i]);
    }
    if (!angles.empty()) {
      o->valid |= MG_METRIC_POOL_EXTENT;
      if (angles.size() == 1) {
        o->pool_angle_min_rad = o->pool_angle_max_rad = angles[0];
      } else {
        sort_angles(&angles);
        float cs, ce, gap;
        largest_gap_cluster_bounds(angles, &cs, &ce, &gap);
        o->pool_angle_min_rad = cs;
        o->pool_angle_max_rad = ce;
      }
    }
    // fluid_free_surface_line, metrics.rs:414-461
    if (pts.size() >= 3) {
      const float n = (float)pts.size();
      Vec2 sum;
      for (const Vec2& p : pts) sum = sum + p;
      const Vec2 c = sum / n;
      float cxx = 0.0f, cyy = 0.0f, cxy = 0.0f;
      for (const Vec2& p : pts) {
        const Vec2 e = p - c;
        cxx += e.x * e.x;
        cyy += e.y * e.y;
        cxy += e.x * e.y;
      }
      cxx /= n;
      cyy /= n;
      cxy /= n;
      const float angle = 0.5f * atan2f_r(2.0f * cxy, cxx - cyy);
      const Vec2 normal(-sinf_r(angle), cosf_r(angle));
      o->valid |= MG_METRIC_FREE_SURFACE;
      o->free_surface_angle_rad = angle;
      o->free_surface_offset_m = c.dot(normal);
    }
    // slurry_pool_depth_at_bottom, metrics.rs:463-477
    const float down = 3.0f * FRAC_PI_2_F;
    bool any = false;
    float min_dist = 0.0f;
    for (size_t i = 0; i < nf; ++i) {
      if (angular_separation(world_angle(f.x[i]), down) <= POOL_DEPTH_BAND_RAD) {
        const float dist = f.x[i].length();
        min_dist = any ? fmin_r(min_dist, dist) : dist;
        any = true;
      }
    }
    if (any) {
      o->valid |= MG_METRIC_POOL_DEPTH;
      o->pool_depth_m = d.radius_m - min_dist;
    }
  }
  // mixing_index, metrics.rs:506-576
  float mi = 0.0f;
  if (mixing_index(f, d, &mi)) {
    o->valid |= MG_METRIC_MIXING;
    o->mixing_index = mi;
  }
  // total_kinetic_energy_j, metrics.rs:581-590
  float ke = 0.0f;
  for (size_t i = 0; i < nb; ++i) ke += 0.5f * b.mass * b.v[i].length_squared() + 0.5f * b.inertia * b.omega[i] * b.omega[i];
  o->total_kinetic_energy_j = ke;
  // max_ball_overlap_fraction, metrics.rs:599-612
  if (nb >= 2 && b.radius > 0.0f) {
    const float r = b.radius;
    UniformGrid g = UniformGrid::build(b.x, fmax_r(2.0f * r * 1.05f, 1e-6f));
    float mo = 0.0f;
    g.for_each_candidate_pair([&](uint32_t i, uint32_t j) {
      const float dist = (b.x[i] - b.x[j]).length();
      const float ov = fmax_r(2.0f * r - dist, 0.0f);
      mo = fmax_r(mo, ov / r);
    });
    o->max_ball_overlap_fraction = mo;
  }
  // max_ball_wall_overlap_fraction, metrics.rs:621-634
  if (nb > 0 && b.radius > 0.0f) {
    const float r = b.radius;
    float mw = 0.0f;
    for (size_t i = 0; i < nb; ++i) mw = fmax_r(mw, fmax_r(r - wall_distance(d, b.x[i], drum_angle), 0.0f) / r);
    o->max_ball_wall_overlap_fraction = mw;
  }
  // fluid density errors, metrics.rs:649-711
  if (nf > 0 && f.rest_density > 0.0f) {
    const std::vector<float> rho = fluid_densities(f);
    const float rest = f.rest_density;
    float mx = 0.0f, sm = 0.0f, cmx = 0.0f, csm = 0.0f;
    for (float v : rho) mx = fmax_r(mx, std::fabs(v - rest) / rest);
    for (float v : rho) sm += std::fabs(v - rest) / rest;
    for (float v : rho) cmx = fmax_r(cmx, fmax_r(v / rest - 1.0f, 0.0f));
    for (float v : rho) csm += fmax_r(v / rest - 1.0f, 0.0f);
    o->valid |= MG_METRIC_DENSITY;
    o->max_fluid_density_error_fraction = mx;
    o->mean_fluid_density_error_fraction = sm / (float)rho.size();
    o->max_fluid_compression_error_fraction = cmx;
    o->mean_fluid_compression_error_fraction = csm / (float)rho.size();
  }
  o->drum_omega_rad_s = d.omega;
  o->fluid_particle_count = (uint32_t)nf;
}

}  // namespace orc
