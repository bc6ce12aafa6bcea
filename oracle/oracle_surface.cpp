// Oracle (test infrastructure only): surface::extract_surface (surface.rs:233-272) and the
// functions it calls (surface.rs:39-218, 279-416), with flatten_polygons (surface.rs:420-430),
// restated in plain C++ over the oracle's state, for checking the device's free-surface kernels.
// The segment chaining keeps the reference's data structures (a segment list in cell order and a
// map from grid edge to the segments touching it, in push order), so it shares no code or layout
// with the device path.
//
// glam 0.29.3 (Cargo.lock) supplies Vec2::lerp, restated here from its published definition:
// lerp(a, b, s) = a * (1 - s) + b * s, per component, without contraction.
//
// Parity status: surface.rs ships property tests only (no golden polygons); the oracle is pinned
// against those properties (tests/test_oracle_surface.py).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../include/millgpu.h"
#include "oracle_core.hpp"

namespace orc {
namespace {

constexpr int GRID = MG_SURFACE_GRID;            // surface.rs:27
constexpr Real SPLAT_RADIUS_FACTOR = Real(1.5);      // surface.rs:29
constexpr Real THRESHOLD_FRACTION = Real(0.5);       // surface.rs:31

// surface.rs:39-46
Real splat_kernel(Real r2, Real radius) {
  const Real radius2 = radius * radius;
  if (r2 >= radius2) return Real(0.0);
  const Real t = Real(1.0) - r2 / radius2;
  return t * t * t;
}

// surface.rs:140-143: round half away from zero, clamp to the grid, NaN casts to 0
int grid_index(Real world, Real drum_radius_m, Real cell_size) {
  Real raw = std::round((world + drum_radius_m) / cell_size);
  if (raw < Real(0.0)) raw = Real(0.0);
  if (raw > (Real)(GRID - 1)) raw = (Real)(GRID - 1);
  return std::isnan(raw) ? 0 : (int)raw;
}

// surface.rs:145-150
Vec2 grid_point(int gi, int gj, Real drum_radius_m, Real cell_size) {
  return Vec2(-drum_radius_m + (Real)gi * cell_size, -drum_radius_m + (Real)gj * cell_size);
}

Vec2 lerp(Vec2 a, Vec2 b, Real s) { return Vec2(a.x * (Real(1.0) - s) + b.x * s, a.y * (Real(1.0) - s) + b.y * s); }

// EdgeId (surface.rs:155-161): kind 0 Horizontal(i, j), kind 1 Vertical(i, j)
struct EdgeId {
  int kind, i, j;
  bool operator==(const EdgeId& o) const { return kind == o.kind && i == o.i && j == o.j; }
};
struct EdgeHash {
  size_t operator()(const EdgeId& e) const {
    return (size_t)e.kind * 1000003u + (size_t)(e.i + 1) * 4099u + (size_t)(e.j + 1);
  }
};

// surface.rs:166-187
Vec2 interp_edge(EdgeId e, const std::vector<Real>& field, Real threshold, Real drum_radius_m,
                 Real cell_size) {
  const int gi0 = e.i, gj0 = e.j;
  const int gi1 = e.kind == 0 ? e.i + 1 : e.i;
  const int gj1 = e.kind == 0 ? e.j : e.j + 1;
  const Real v0 = field[gj0 * GRID + gi0];
  const Real v1 = field[gj1 * GRID + gi1];
  Real t;
  if (std::fabs(v1 - v0) > Real(1e-9)) {
    t = (threshold - v0) / (v1 - v0);
    if (t < Real(0.0)) t = Real(0.0);
    if (t > Real(1.0)) t = Real(1.0);
  } else {
    t = Real(0.5);
  }
  return lerp(grid_point(gi0, gj0, drum_radius_m, cell_size), grid_point(gi1, gj1, drum_radius_m, cell_size), t);
}

// surface.rs:194-207: (count, pairs) per case
int cell_edge_pairs(int c, int pairs[2][2]) {
  auto set = [&](int k, int a, int b) { pairs[k][0] = a; pairs[k][1] = b; };
  switch (c) {
    case 1: case 14: set(0, 3, 0); return 1;
    case 2: case 13: set(0, 0, 1); return 1;
    case 3: case 12: set(0, 3, 1); return 1;
    case 4: case 11: set(0, 1, 2); return 1;
    case 6: case 9: set(0, 0, 2); return 1;
    case 7: case 8: set(0, 3, 2); return 1;
    case 5: set(0, 3, 0); set(1, 1, 2); return 2;
    case 10: set(0, 0, 1); set(1, 3, 2); return 2;
    default: return 0;
  }
}

// surface.rs:209-218
EdgeId cell_edge_id(int ci, int cj, int side) {
  switch (side) {
    case 0: return EdgeId{0, ci, cj};
    case 1: return EdgeId{1, ci + 1, cj};
    case 2: return EdgeId{0, ci, cj + 1};
    default: return EdgeId{1, ci, cj};
  }
}

using Segments = std::vector<std::pair<EdgeId, EdgeId>>;
using ByEdge = std::unordered_map<EdgeId, std::vector<size_t>, EdgeHash>;

// surface.rs:371-399
void extend_chain(std::vector<EdgeId>* chain, const Segments& segs, const ByEdge& by_edge,
                  std::vector<char>* visited, bool forward) {
  for (;;) {
    const EdgeId tip = forward ? chain->back() : chain->front();
    auto it = by_edge.find(tip);
    if (it == by_edge.end()) return;
    size_t next = SIZE_MAX;
    for (size_t idx : it->second)
      if (!(*visited)[idx]) { next = idx; break; }
    if (next == SIZE_MAX) return;
    (*visited)[next] = 1;
    const EdgeId other = segs[next].first == tip ? segs[next].second : segs[next].first;
    if (forward) chain->push_back(other);
    else chain->insert(chain->begin(), other);
  }
}

// surface.rs:403-416
std::vector<Vec2> chaikin_smooth_closed(const std::vector<Vec2>& pts) {
  if (pts.size() < 3) return pts;
  const size_t n = pts.size();
  std::vector<Vec2> out;
  out.reserve(2 * n);
  for (size_t i = 0; i < n; ++i) {
    const Vec2 p0 = pts[i], p1 = pts[(i + 1) % n];
    out.push_back(lerp(p0, p1, Real(0.25)));
    out.push_back(lerp(p0, p1, Real(0.75)));
  }
  return out;
}

// surface.rs:359-366
Vec2 project_inside_wall(Vec2 p, const Drum& drum, Real drum_angle) {
  Real d;
  Vec2 n;
  drum.sdf_world(p, drum_angle, &d, &n);
  return d < Real(0.0) ? p - d * n : p;
}

// surface.rs:279-351
std::vector<std::vector<Vec2>> polygons_at_threshold(const std::vector<Real>& field, Real threshold,
                                                     Real drum_radius_m, Real cell_size, const Drum& drum,
                                                     Real drum_angle) {
  Segments segs;
  for (int cj = 0; cj < GRID - 1; ++cj)
    for (int ci = 0; ci < GRID - 1; ++ci) {
      auto corner = [&](int di, int dj) { return field[(cj + dj) * GRID + (ci + di)] > threshold ? 1 : 0; };
      const int c = corner(0, 0) | corner(1, 0) << 1 | corner(1, 1) << 2 | corner(0, 1) << 3;
      int pairs[2][2];
      const int np = cell_edge_pairs(c, pairs);
      for (int k = 0; k < np; ++k) segs.emplace_back(cell_edge_id(ci, cj, pairs[k][0]), cell_edge_id(ci, cj, pairs[k][1]));
    }
  if (segs.empty()) return {};
  ByEdge by_edge;
  for (size_t idx = 0; idx < segs.size(); ++idx) {
    by_edge[segs[idx].first].push_back(idx);
    by_edge[segs[idx].second].push_back(idx);
  }
  std::vector<char> visited(segs.size(), 0);
  std::vector<std::vector<EdgeId>> chains;
  for (size_t start = 0; start < segs.size(); ++start) {
    if (visited[start]) continue;
    visited[start] = 1;
    std::vector<EdgeId> chain{segs[start].first, segs[start].second};
    extend_chain(&chain, segs, by_edge, &visited, true);
    extend_chain(&chain, segs, by_edge, &visited, false);
    if (chain.size() > 1 && chain.front() == chain.back()) chain.pop_back();
    chains.push_back(std::move(chain));
  }
  std::vector<std::vector<Vec2>> polys;
  for (const auto& chain : chains) {
    std::vector<Vec2> pts;
    for (const EdgeId& e : chain) pts.push_back(interp_edge(e, field, threshold, drum_radius_m, cell_size));
    std::vector<Vec2> sm = chaikin_smooth_closed(pts);
    for (Vec2& p : sm) p = project_inside_wall(p, drum, drum_angle);
    polys.push_back(std::move(sm));
  }
  return polys;
}

}  // namespace

// surface.rs:71-74
Real surface_phi_full(const Fluid& f) {
  const Real splat_radius = SPLAT_RADIUS_FACTOR * f.h;
  const Real number_density = f.rest_density / fmax_r(f.particle_mass, Real(1e-12));
  return number_density * (PI_F * splat_radius * splat_radius / Real(4.0));
}

// surface.rs:84-131
std::vector<Real> surface_build_field(const Fluid& f, const Drum& drum, Real drum_angle) {
  const Real drum_radius_m = drum.radius_m;
  std::vector<Real> field((size_t)GRID * GRID, Real(0.0));
  if (f.len() == 0 || drum_radius_m <= Real(0.0)) return field;
  const Real splat_radius = SPLAT_RADIUS_FACTOR * f.h;
  const Real cell_size = Real(2.0) * drum_radius_m / ((Real)GRID - Real(1.0));
  for (const Vec2& p : f.x) {
    const int gi_min = grid_index(p.x - splat_radius, drum_radius_m, cell_size);
    const int gi_max = grid_index(p.x + splat_radius, drum_radius_m, cell_size);
    const int gj_min = grid_index(p.y - splat_radius, drum_radius_m, cell_size);
    const int gj_max = grid_index(p.y + splat_radius, drum_radius_m, cell_size);
    for (int gj = gj_min; gj <= gj_max; ++gj)
      for (int gi = gi_min; gi <= gi_max; ++gi) {
        const Vec2 gp = grid_point(gi, gj, drum_radius_m, cell_size);
        field[(size_t)gj * GRID + gi] += splat_kernel((gp - p).length_squared(), splat_radius);
      }
  }
  const Vec2 to_local = Vec2::from_angle(-drum_angle);
  for (int gj = 0; gj < GRID; ++gj)
    for (int gi = 0; gi < GRID; ++gi) {
      Real& v = field[(size_t)gj * GRID + gi];
      if (v == Real(0.0)) continue;
      if (drum.sdf(rotate(grid_point(gi, gj, drum_radius_m, cell_size), to_local)) < Real(0.0)) v = Real(0.0);
    }
  return field;
}

// surface.rs:233-272 followed by surface.rs:420-430
std::vector<Real> surface_extract_flat(const Fluid& f, const Drum& drum, Real drum_angle) {
  std::vector<std::vector<Vec2>> polys;
  const Real drum_radius_m = drum.radius_m;
  if (f.len() != 0 && drum_radius_m > Real(0.0)) {
    const std::vector<Real> field = surface_build_field(f, drum, drum_angle);
    const Real cell_size = Real(2.0) * drum_radius_m / ((Real)GRID - Real(1.0));
    polys = polygons_at_threshold(field, THRESHOLD_FRACTION * surface_phi_full(f), drum_radius_m, cell_size, drum,
                                  drum_angle);
    if (polys.empty()) {
      Real peak = Real(0.0);
      for (Real v : field) peak = fmax_r(peak, v);
      if (peak > Real(0.0))
        polys = polygons_at_threshold(field, THRESHOLD_FRACTION * peak, drum_radius_m, cell_size, drum, drum_angle);
    }
  }
  std::vector<Real> out{(Real)polys.size()};
  for (const auto& poly : polys) {
    out.push_back((Real)poly.size());
    for (const Vec2& p : poly) {
      out.push_back(p.x);
      out.push_back(p.y);
    }
  }
  return out;
}

}  // namespace orc
