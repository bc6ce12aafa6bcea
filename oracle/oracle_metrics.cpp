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

constexpr Real WALL_MARGIN_BALL_RADII = Real(2.5);                 // metrics.rs:37
constexpr size_t MIN_WALL_BALLS = 6;                           // metrics.rs:41
constexpr Real CENTRIFUGE_GAP_THRESHOLD_RAD = PI_F * Real(0.3);    // metrics.rs:45
constexpr Real POOL_WALL_MARGIN_H = Real(1.5);                     // metrics.rs:48
constexpr Real POOL_DEPTH_BAND_RAD = Real(5.0) * PI_F / Real(180.0);    // metrics.rs:51
constexpr Real FRAC_PI_2_F = Real(1.57079632679489661923);

Real wall_distance(const Drum& d, Vec2 p, Real drum_angle) {
  Real dist;
  Vec2 nrm;
  d.sdf_world(p, drum_angle, &dist, &nrm);
  return dist;
}

// metrics.rs:281-284
Real angular_separation(Real a, Real b) {
  Real d = rem_euclid_r(a - b, TAU_F);
  return fmin_r(d, TAU_F - d);
}

// metrics.rs:292-307 over angles sorted ascending (n >= 2)
void largest_gap_cluster_bounds(const std::vector<Real>& a, Real* start, Real* end, Real* gap) {
  const size_t n = a.size();
  Real max_gap = a[0] + TAU_F - a[n - 1];
  size_t gap_k = n - 1;
  for (size_t i = 0; i + 1 < n; ++i) {
    Real g = a[i + 1] - a[i];
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
void sort_angles(std::vector<Real>* a) {
  std::stable_sort(a->begin(), a->end(), [](Real x, Real y) { return x < y; });
}

Real world_angle(Vec2 p) { return rem_euclid_r(atan2f_r(p.y, p.x), TAU_F); }

}  // namespace

// metrics.rs:195-273 (the fields compute fills)
void metrics_compute(const Balls& b, const Fluid& f, const Drum& d, Real drum_angle, MgMetrics* o) {
  std::memset(o, 0, sizeof(*o));
  const size_t nb = b.len(), nf = f.len();
  // charge_toe_shoulder, metrics.rs:327-360
  if (nb > 0) {
    const Real margin = WALL_MARGIN_BALL_RADII * b.radius;
    std::vector<Real> angles;
    for (size_t i = 0; i < nb; ++i)
      if (wall_distance(d, b.x[i], drum_angle) < margin) angles.push_back(world_angle(b.x[i]));
    if (angles.size() >= MIN_WALL_BALLS) {
      sort_angles(&angles);
      Real cs, ce, gap;
      largest_gap_cluster_bounds(angles, &cs, &ce, &gap);
      if (!(gap <= CENTRIFUGE_GAP_THRESHOLD_RAD)) {
        o->valid |= MG_METRIC_TOE_SHOULDER;
        o->toe_angle_rad = d.omega >= Real(0.0) ? cs : ce;
        o->shoulder_angle_rad = d.omega >= Real(0.0) ? ce : cs;
      }
    }
    // charge_centroid, metrics.rs:362-369
    Vec2 sum;
    for (size_t i = 0; i < nb; ++i) sum = sum + b.x[i];
    const Vec2 c = sum / (Real)nb;
    o->valid |= MG_METRIC_CENTROID;
    o->charge_centroid_m[0] = c.x;
    o->charge_centroid_m[1] = c.y;
  }
  if (nf > 0) {
    const Real margin = POOL_WALL_MARGIN_H * f.h;
    // slurry_pool_angular_extent, metrics.rs:377-400
    std::vector<Real> angles;
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
        Real cs, ce, gap;
        largest_gap_cluster_bounds(angles, &cs, &ce, &gap);
        o->pool_angle_min_rad = cs;
        o->pool_angle_max_rad = ce;
      }
    }
    // fluid_free_surface_line, metrics.rs:414-461
    if (pts.size() >= 3) {
      const Real n = (Real)pts.size();
      Vec2 sum;
      for (const Vec2& p : pts) sum = sum + p;
      const Vec2 c = sum / n;
      Real cxx = Real(0.0), cyy = Real(0.0), cxy = Real(0.0);
      for (const Vec2& p : pts) {
        const Vec2 e = p - c;
        cxx += e.x * e.x;
        cyy += e.y * e.y;
        cxy += e.x * e.y;
      }
      cxx /= n;
      cyy /= n;
      cxy /= n;
      const Real angle = Real(0.5) * atan2f_r(Real(2.0) * cxy, cxx - cyy);
      const Vec2 normal(-sinf_r(angle), cosf_r(angle));
      o->valid |= MG_METRIC_FREE_SURFACE;
      o->free_surface_angle_rad = angle;
      o->free_surface_offset_m = c.dot(normal);
    }
    // slurry_pool_depth_at_bottom, metrics.rs:463-477
    const Real down = Real(3.0) * FRAC_PI_2_F;
    bool any = false;
    Real min_dist = Real(0.0);
    for (size_t i = 0; i < nf; ++i) {
      if (angular_separation(world_angle(f.x[i]), down) <= POOL_DEPTH_BAND_RAD) {
        const Real dist = f.x[i].length();
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
  Real mi = Real(0.0);
  if (mixing_index(f, d, &mi)) {
    o->valid |= MG_METRIC_MIXING;
    o->mixing_index = mi;
  }
  // total_kinetic_energy_j, metrics.rs:581-590
  Real ke = Real(0.0);
  for (size_t i = 0; i < nb; ++i) ke += Real(0.5) * b.mass * b.v[i].length_squared() + Real(0.5) * b.inertia * b.omega[i] * b.omega[i];
  o->total_kinetic_energy_j = ke;
  // max_ball_overlap_fraction, metrics.rs:599-612
  if (nb >= 2 && b.radius > Real(0.0)) {
    const Real r = b.radius;
    UniformGrid g = UniformGrid::build(b.x, fmax_r(Real(2.0) * r * Real(1.05), Real(1e-6)));
    Real mo = Real(0.0);
    g.for_each_candidate_pair([&](uint32_t i, uint32_t j) {
      const Real dist = (b.x[i] - b.x[j]).length();
      const Real ov = fmax_r(Real(2.0) * r - dist, Real(0.0));
      mo = fmax_r(mo, ov / r);
    });
    o->max_ball_overlap_fraction = mo;
  }
  // max_ball_wall_overlap_fraction, metrics.rs:621-634
  if (nb > 0 && b.radius > Real(0.0)) {
    const Real r = b.radius;
    Real mw = Real(0.0);
    for (size_t i = 0; i < nb; ++i) mw = fmax_r(mw, fmax_r(r - wall_distance(d, b.x[i], drum_angle), Real(0.0)) / r);
    o->max_ball_wall_overlap_fraction = mw;
  }
  // fluid density errors, metrics.rs:649-711
  if (nf > 0 && f.rest_density > Real(0.0)) {
    const std::vector<Real> rho = fluid_densities(f);
    const Real rest = f.rest_density;
    Real mx = Real(0.0), sm = Real(0.0), cmx = Real(0.0), csm = Real(0.0);
    for (Real v : rho) mx = fmax_r(mx, std::fabs(v - rest) / rest);
    for (Real v : rho) sm += std::fabs(v - rest) / rest;
    for (Real v : rho) cmx = fmax_r(cmx, fmax_r(v / rest - Real(1.0), Real(0.0)));
    for (Real v : rho) csm += fmax_r(v / rest - Real(1.0), Real(0.0));
    o->valid |= MG_METRIC_DENSITY;
    o->max_fluid_density_error_fraction = mx;
    o->mean_fluid_density_error_fraction = sm / (Real)rho.size();
    o->max_fluid_compression_error_fraction = cmx;
    o->mean_fluid_compression_error_fraction = csm / (Real)rho.size();
  }
  o->drum_omega_rad_s = d.omega;
  o->fluid_particle_count = (uint32_t)nf;
}

}  // namespace orc
