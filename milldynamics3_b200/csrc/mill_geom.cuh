// Drum geometry on the device (geometry.rs:37-275): circle plus trapezoid-lifter SDF in the drum
// frame, the world-space query with its central-difference normal (EPS = 1e-4), the wall
// velocity and the swept time of impact. Lifter frames and the drum-angle rotations arrive
// precomputed in the StepUniform (host trig), so the per-query work is pure f32 arithmetic.
#pragma once

#include "mill_common.cuh"

namespace mg {

// geometry.rs:258-275 convex_polygon_sdf over the 4 CCW vertices of one lifter.
__device__ __forceinline__ float convex_quad_sdf(V2 p, const V2* verts) {
  float min_dist_sq = 3.40282347e38f;
  bool inside = true;
  for (int i = 0; i < 4; ++i) {
    V2 a = verts[i];
    V2 b = verts[(i + 1) & 3];
    V2 edge = b - a;
    V2 to_p = p - a;
    float len_sq = edge.len2();
    if (len_sq < 1e-12f) continue;
    float t = clamp_r(to_p.dot(edge) / len_sq, 0.0f, 1.0f);
    V2 closest = a + edge * t;
    min_dist_sq = fmin_r(min_dist_sq, (p - closest).len2());
    float cross = edge.x * to_p.y - edge.y * to_p.x;
    if (cross < 0.0f) inside = false;
  }
  float dist = sqrtf(min_dist_sq);
  return inside ? dist : -dist;
}

// geometry.rs:37-72 Drum::sdf (local frame)
__device__ __forceinline__ float drum_sdf(const StepUniform& U, V2 p) {
  float d = U.drum_radius - p.len();
  if (U.lifter_count == 0) return d;
  float r = U.drum_radius;
  float r_top = r - U.lifter_height;
  V2 verts[4] = {V2(r, -U.lifter_base_half), V2(r, U.lifter_base_half), V2(r_top, U.lifter_top_half),
                 V2(r_top, -U.lifter_top_half)};
  // A lifter whose distance certainly exceeds the circle term d cannot change fmin(d, -max_inside)
  // (fmin and fmax only select), so it is skipped. A proper CCW quad (0 < h < R, b, t > 0) lies in
  // the disk of centre (R - h/2, 0) and radius rho = sqrt(h^2/4 + max(b, t)^2) of its frame, and
  // its convex_quad_sdf is then minus the distance for points outside it; the lifter is skipped
  // when the point is farther than d + rho from the centre, with margins (1e-4 R in the reach,
  // 2e-6 R and a relative 1e-5 in the comparison) far above the f32 rounding of either side.
  const bool cull = U.lifter_height > 0.0f && U.lifter_height < r && U.lifter_base_half > 0.0f &&
                    U.lifter_top_half > 0.0f;
  const float cx = r - 0.5f * U.lifter_height;
  const float wmax = fmaxf(U.lifter_base_half, U.lifter_top_half);
  const float rho = sqrtf(0.25f * U.lifter_height * U.lifter_height + wmax * wmax);
  const float reach = d + rho * 1.00001f + 1e-4f * r;
  const float far2 = (reach + 2e-6f * r) * (reach + 2e-6f * r) * 1.00001f;
  float max_inside = -INFINITY;
  for (uint32_t k = 0; k < U.lifter_count; ++k) {
    float s = U.lifter_sin[k], c = U.lifter_cos[k];
    float pr = p.x * c + p.y * s;
    float pt = -p.x * s + p.y * c;
    if (cull && reach > 0.0f && (pr - cx) * (pr - cx) + pt * pt > far2) continue;
    max_inside = fmax_r(max_inside, convex_quad_sdf(V2(pr, pt), verts));
  }
  return fmin_r(d, -max_inside);
}

// geometry.rs:87-109 Drum::sdf_world with the rotations from_angle(-angle) / from_angle(angle).
__device__ __forceinline__ void drum_sdf_world(const StepUniform& U, V2 pw, V2 to_local, V2 to_world, float& d,
                                               V2& normal) {
  if (!pw.finite()) { d = 0.0f; normal = V2(); return; }
  V2 pl = rotate(pw, to_local);
  const float EPS = 1e-4f;
  float dd = drum_sdf(U, pl);
  float gx = drum_sdf(U, pl + V2(EPS, 0.0f)) - drum_sdf(U, pl - V2(EPS, 0.0f));
  float gy = drum_sdf(U, pl + V2(0.0f, EPS)) - drum_sdf(U, pl - V2(0.0f, EPS));
  V2 grad = V2(gx, gy) / (2.0f * EPS);
  V2 nl = grad.len2() > 1e-12f ? grad.normalize() : -pl.normalize_or_zero();
  d = dd;
  normal = rotate(nl, to_world);
}

// drum_sdf_world in two halves, for callers that need the normal only in contact: the distance
// (one SDF evaluation; pl receives the local point) and then the normal at the same point. Same
// values as drum_sdf_world, including d = 0 and a zero normal for a non-finite point.
__device__ __forceinline__ float drum_sdf_world_dist(const StepUniform& U, V2 pw, V2 to_local, V2& pl) {
  if (!pw.finite()) { pl = V2(); return 0.0f; }
  pl = rotate(pw, to_local);
  return drum_sdf(U, pl);
}

__device__ __forceinline__ V2 drum_sdf_world_normal(const StepUniform& U, V2 pw, V2 pl, V2 to_world) {
  if (!pw.finite()) return V2();
  const float EPS = 1e-4f;
  float gx = drum_sdf(U, pl + V2(EPS, 0.0f)) - drum_sdf(U, pl - V2(EPS, 0.0f));
  float gy = drum_sdf(U, pl + V2(0.0f, EPS)) - drum_sdf(U, pl - V2(0.0f, EPS));
  V2 grad = V2(gx, gy) / (2.0f * EPS);
  V2 nl = grad.len2() > 1e-12f ? grad.normalize() : -pl.normalize_or_zero();
  return rotate(nl, to_world);
}

// True when the f32 drum SDF at the local point pl is certainly >= bound, decided without
// evaluating the lifters. Every point q of a lifter quad (R, -b), (R, b), (R - h, t), (R - h, -t)
// with 0 < h < R and b, t > 0 has |q| >= R - h, so the circle term and each lifter term are both
// at least (R - h) - |pl| in exact arithmetic; the margin (1e-4 R) exceeds the f32 rounding of the
// full evaluation by orders of magnitude. False (evaluate in full) for other lifter shapes and for
// non-finite points.
__device__ __forceinline__ bool drum_sdf_clear(const StepUniform& U, V2 pl, float bound) {
  double inner = (double)U.drum_radius;
  if (U.lifter_count != 0) {
    if (!(U.lifter_height > 0.0f && U.lifter_height < U.drum_radius && U.lifter_base_half > 0.0f &&
          U.lifter_top_half > 0.0f))
      return false;
    inner -= (double)U.lifter_height;
  }
  const double pr = sqrt((double)pl.x * (double)pl.x + (double)pl.y * (double)pl.y);
  return inner - pr >= (double)bound + 1e-4 * (double)U.drum_radius;
}

__device__ __forceinline__ V2 wall_velocity(float omega, V2 p) { return omega * V2(-p.y, p.x); }

// geometry.rs:146-194 Drum::toi_swept; returns false for None.
__device__ inline bool drum_toi_swept(const StepUniform& U, V2 x0, V2 x1, float a0, float a1, float radius, float& t_out) {
  V2 local0 = rotate(x0, U.to_local0);
  if (drum_sdf(U, local0) - radius <= 0.0f) return false;
  V2 path = x1 - x0;
  float path_len = path.len();
  float dangle = a1 - a0;
  float pos_bound = x0.len() + path_len;
  float bound = path_len + fabsf(dangle) * pos_bound;
  if (bound < 1e-9f) return false;
  float t = 0.0f;
  for (int it = 0; it < 32; ++it) {
    float angle_t = a0 + dangle * t;
    V2 x_t = x0 + path * t;
    float na = -angle_t;
    V2 local = rotate(x_t, V2(cosf_r(na), sinf_r(na)));
    float d = drum_sdf(U, local) - radius;
    if (d <= 0.0f) { t_out = t; return true; }
    float step_t = fmax_r(d / bound, 1e-6f);
    t += step_t;
    if (t >= 1.0f) return false;
  }
  t_out = fmin_r(t, 1.0f);
  return true;
}

}  // namespace mg
