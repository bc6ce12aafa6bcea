// The fluid half of the sub-step (FluidParticles::step_coupled, pbf.rs:1174-2365) for one mill,
// executed by one thread block. Per-particle and per-ball stages are block-stride loops in
// gather form (no atomics on positions); the reference's order-dependent reductions and its
// Gauss-Seidel sweeps (drag, buoyancy) are replayed in the reference order, so the results match
// the sequential Rust arithmetic bit for bit.
#pragma once

#include "mill_geom.cuh"
#include "mill_grid.cuh"
#include "mill_replay.cuh"
#include "mill_wide.cuh"

namespace mg {

constexpr float EPSILON_RELAX = 200.0f;
constexpr uint32_t ADAPTIVE_MAX_EXTRA = 6;
constexpr float COMPRESSION_TOL = 0.02f;
constexpr float OVERLAP_PUSH_MARGIN = 0.05f;
constexpr float VISC_CG_TOL = 1e-3f;
constexpr uint32_t VISC_CG_MAX = 50;
constexpr float VISC_ETA = 0.01f;
constexpr float CENTRAL_VISC = 4.0f;
constexpr float BALL_BC_GAIN = 0.5f;

struct FluidShared {
  GridHdr hA, hB, hBall;
  uint32_t n_edges, n_recs, n_groups, n_links, links_in_range;
  float fscal[8];
  double dscal[8];
  uint32_t uscal[8];
};

__device__ __forceinline__ float fluid_vmax(const StepUniform& U) {
  return 5.0f * (fabsf(U.drum_omega) * U.drum_radius + sqrtf(4.0f * fabsf(GRAVITY) * U.drum_radius));
}

// pbf.rs:924-926: 0.5 m sum |v|^2 in f64, summed in particle order.
static __device__ __noinline__ double kinetic_energy_seq(const float2* v, uint32_t n, float mass, FluidShared& S) {
  if (tid() < 32) {
    double s = warp_ordered_sum(0.0, n, [&](uint32_t i, double& t) { t = (double)V2(v[i]).len2(); return true; });
    if (tid() == 0) S.dscal[7] = 0.5 * (double)mass * s;
  }
  __syncthreads();
  double r = S.dscal[7];
  __syncthreads();
  return r;
}

// pbf.rs:292-294 dot in the reference's sequential f32 order, or in f64 (deterministic tree).
static __device__ __noinline__ double block_dot(const float2* a, const float2* b, uint32_t len, bool fp64, FluidShared& S) {
  if (fp64) {
    double acc = 0.0;
    for (uint32_t e = tid(); e < len; e += nthr())
      acc += (double)a[e].x * (double)b[e].x + (double)a[e].y * (double)b[e].y;
    return block_sum_d(acc);
  }
  return (double)block_seq_sum_f32(0.0f, len, [&](uint32_t e) { return V2(a[e]).dot(V2(b[e])); });
}

// pbf.rs:738-744 residual norm sqrt(sum inv_diag |r|^2), sequential f32 or f64.
static __device__ __noinline__ double block_res_norm(const float2* r, const float* inv, uint32_t len, bool fp64, FluidShared& S) {
  if (fp64) {
    double acc = 0.0;
    for (uint32_t e = tid(); e < len; e += nthr())
      acc += (double)inv[e] * ((double)r[e].x * (double)r[e].x + (double)r[e].y * (double)r[e].y);
    return sqrt(block_sum_d(acc));
  }
  return (double)sqrtf(block_seq_sum_f32(0.0f, len, [&](uint32_t e) { return inv[e] * V2(r[e]).len2(); }));
}

// pbf.rs:359-377 laplacian row i.
__device__ __forceinline__ V2 laplacian_row(const MillDev& m, const float2* v, uint32_t i) {
  V2 sum;
  V2 vi(v[i]);
  const uint32_t k0 = m.nbr_off[i], k1 = m.nbr_off[i + 1];
#pragma unroll 4
  for (uint32_t k = k0; k < k1; ++k) {
    uint32_t j = m.nbrs[k];
    V2 e(m.visc_dir[k]);
    sum += (CENTRAL_VISC * m.visc_w[k] * e.dot(vi - V2(v[j]))) * e;
  }
  return sum;
}

// pbf.rs:544-625 squeeze-film coefficient pieces (f64, mac/lubrication.rs:49-115)
__device__ __forceinline__ double film_coefficient(const FilmConsts& f, double h) {
  double eps = h / f.r;
  return f.prefactor / (h * sqrt(h)) * (1.0 + f.c1 * eps + f.c2 * eps * eps);
}
__device__ __forceinline__ double resolved_ratio(double hc) {
  const double T0[6] = {0.0, 0.5, 1.0, 2.0, 4.0, 8.0};
  const double T1[6] = {0.0, 0.06, 0.25, 0.90, 0.99, 1.0};
  if (hc >= 8.0) return 1.0;
  double h = hc < 0.0 ? 0.0 : hc;
  if (hc != hc) h = 0.0;
  for (int k = 0; k < 5; ++k) {
    if (h <= T0[k + 1]) {
      double t = (h - T0[k]) / (T0[k + 1] - T0[k]);
      return T1[k] + t * (T1[k + 1] - T1[k]);
    }
  }
  return 1.0;
}

// One squeeze link candidate (ball i, partner j or wall); returns false when not in range.
struct LinkEval { bool in_range, emit; V2 n; float c; };

// Ball i at xi with viscous start velocity v0i against ball j (xj, v0j).
__device__ __forceinline__ LinkEval link_pair(const MillDev& m, const StepUniform& U, V2 xi, V2 v0i, V2 xj, V2 v0j,
                                              float reach, float range2, double dxd, float c_max, bool need_c = true) {
  LinkEval L{false, false, V2(), 0.0f};
  float r = m.b_r;
  V2 e = xj - xi;
  if (e.len2() >= range2 || !e.finite()) return L;
  float dist = e.len();
  float gap = dist - 2.0f * r;
  if (gap >= reach || dist < 1e-9f) return L;
  L.in_range = true;
  L.n = e / dist;
  if (L.n.dot(v0i - v0j) <= 0.0f) return L;
  L.emit = true;
  if (!need_c) return L;
  double weight = 1.0 - resolved_ratio((double)gap / dxd);
  double hh = (double)gap > 0.02 * (double)r ? (double)gap : 0.02 * (double)r;
  double c = weight * film_coefficient(U.pair_film, hh);
  L.emit = true;
  L.c = fmin_r(1.0f * (float)c, c_max);
  return L;
}
__device__ __forceinline__ LinkEval link_wall(const MillDev& m, const StepUniform& U, uint32_t i, float reach,
                                              double dxd, float c_max) {
  LinkEval L{false, false, V2(), 0.0f};
  float r = m.b_r;
  V2 xi(m.bx[i]);
  float dist = xi.len();
  float gap = U.drum_radius - r - dist;
  if (!(gap < reach && dist > 1e-9f)) return L;
  L.in_range = true;
  L.n = xi / dist;
  if (L.n.dot(V2(m.ball_v0[i])) <= 0.0f) return L;
  double weight = 1.0 - resolved_ratio((double)gap / dxd);
  double hh = (double)gap > 0.02 * (double)r ? (double)gap : 0.02 * (double)r;
  double c = weight * film_coefficient(U.wall_film, hh);
  L.emit = true;
  L.c = fmin_r(1.0f * (float)c, c_max);
  return L;
}

// Rows t0, t0 + stride, ... of the joint-system operator of pbf.rs:703-737 applied to xx, written
// to out: fluid rows 0..n-1 (Laplacian, then the boundary groups), then ball rows n..n+nb-1
// (linear and angular).
static __device__ void joint_apply_rows(const MillDev& m, float dt, const float2* xx, float2* out, uint32_t t0,
                                 uint32_t stride) {
  const uint32_t n = m.nf, nb = m.nb;
  const float mass = m.f_mass;
  const float k = dt * mass;
  // fluid rows 0..n-1, one thread per row (the loops are unrolled so that the independent loads
  // of consecutive terms overlap; the additions keep their order)
  for (uint32_t t = t0; t < n; t += stride) {
    {
      const uint32_t i = t;
      const V2 lv(laplacian_row(m, xx, i).f2());
      V2 o = mass * (V2(xx[i]) + dt * lv);
      const uint32_t q0 = m.fg_start[i], q1 = m.fg_start[i + 1];
#pragma unroll 4
      for (uint32_t q = q0; q < q1; ++q) {
        uint32_t g = m.fg_list[q];
        uint32_t bi = m.g_ball[g];
        V2 vb(xx[n + bi]);
        float w = xx[n + nb + bi].x;
        V2 rel = V2(xx[i]) - vb;
        V2 lc(m.g_lc[g]);
        V2 d = k * (m.g_c[g] * rel - w * V2(-lc.y, lc.x));
        o += d;
      }
      out[i] = o.f2();
    }
  }
  // ball rows n..n+nb-1, one warp per row: the lanes form the terms of 32 consecutive entries of
  // the row (its groups, then the links naming it as the other ball, then its own links) in
  // parallel, and the three running sums add them in entry order (lane_seq_sum3; o -= d as
  // o + (-d), the same f32 result; entries without an angular term add -0.0, which changes nothing)
  const uint32_t lane = tid() & 31u;
  for (uint32_t bi = t0 >> 5; bi < nb; bi += stride >> 5) {
    const V2 vb(xx[n + bi]);
    const float w = xx[n + nb + bi].x;
    float ox = 0.0f, oy = 0.0f, oa = 0.0f;
    {
      const V2 o0 = m.b_m * vb;
      ox = o0.x;
      oy = o0.y;
      oa = m.b_I * w;
    }
    const uint32_t g0 = m.g_off[bi], ng = m.g_off[bi + 1] - g0;
    const uint32_t lq0 = m.lo_start[bi], nlo = m.lo_start[bi + 1] - lq0;
    const uint32_t l0 = m.l_off[bi], nown = m.l_off[bi + 1] - l0;
    const uint32_t cnt = ng + nlo + nown;
    for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
      const uint32_t e = c0 + lane;
      float tx = -0.0f, ty = -0.0f, ta = -0.0f;
      if (e < ng) {
        const uint32_t g = g0 + e;
        const uint32_t i = m.g_fluid[g];
        const V2 rel = V2(xx[i]) - vb;
        const V2 lc(m.g_lc[g]);
        const V2 d = k * (m.g_c[g] * rel - w * V2(-lc.y, lc.x));
        tx = -d.x;
        ty = -d.y;
        ta = -(k * (cross2(lc, rel) - w * m.g_l2[g]));
      } else if (e < ng + nlo) {
        const uint32_t l = m.lo_list[lq0 + (e - ng)];
        const V2 rel = V2(xx[n + m.l_ball[l]]) - vb;
        const V2 ln(m.l_n[l]);
        const V2 d = (dt * m.l_c[l] * ln.dot(rel)) * ln;
        tx = -d.x;
        ty = -d.y;
      } else if (e < cnt) {
        const uint32_t l = l0 + (e - ng - nlo);
        const uint32_t other = m.l_other[l];
        V2 rel = vb;
        if (other != NONE) rel = rel - V2(xx[n + other]);
        const V2 ln(m.l_n[l]);
        const V2 d = (dt * m.l_c[l] * ln.dot(rel)) * ln;
        tx = d.x;
        ty = d.y;
      }
      lane_seq_sum3(ox, oy, oa, tx, ty, ta, min(32u, cnt - c0));
    }
    if (lane == 0) {
      out[n + bi] = make_float2(ox, oy);
      out[n + nb + bi] = make_float2(oa, 0.0f);
    }
  }
}

// The joint-system operator over all of the mill's blocks (all rows written on return).
static __device__ void joint_apply(const MillDev& m, float dt, const float2* xx, float2* out) {
  wide_phase(m, WIDE_JOINT_APPLY, nullptr, xx, out, [&](uint32_t w0, uint32_t nw) {
    joint_apply_rows(m, dt, xx, out, w0 * 32u + (tid() & 31u), nw * 32u);
  });
}

// Rows t0, t0 + stride, ... of the joint solve's set-up (pbf.rs:641-700): the start vector x, the
// right-hand side and the Jacobi diagonal, fluid rows then ball rows.
static __device__ void cg_setup_rows(const MillDev& m, float dt, uint32_t t0, uint32_t stride) {
  const uint32_t n = m.nf, nb = m.nb;
  const float mass = m.f_mass;
  const float2* V = m.fv;
  float2 *x = m.cg_x, *bvec = m.cg_b;
  float* diag = m.cg_diag;
  const bool use_guess = *m.guess_valid_dev != 0;
  // fluid rows 0..n-1, one thread per row
  for (uint32_t t = t0; t < n; t += stride) {
    const uint32_t i = t;
    V2 v(V[i]);
    x[i] = (use_guess ? v + V2(m.fguess[i]) : v).f2();
    bvec[i] = (mass * v).f2();
    float sw = 0.0f;
    for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) sw += m.visc_w[k];
    float d = mass * (1.0f + dt * (0.5f * CENTRAL_VISC * sw));
    for (uint32_t q = m.fg_start[i]; q < m.fg_start[i + 1]; ++q) d += dt * mass * m.g_c[m.fg_list[q]];
    diag[i] = d;
    m.dv_tmp[i] = V[i];  // v_in for the warm start of the next sub-step
  }
  // ball rows, one warp per ball: the diagonal's terms (groups, then the links naming the ball as
  // the other ball, then its own links) formed by the lanes in parallel and added in entry order
  // by the three-way lane sum (link entries add -0.0 to the angular diagonal: no change)
  const uint32_t lane = tid() & 31u;
  for (uint32_t b = t0 >> 5; b < nb; b += stride >> 5) {
    V2 v0(m.ball_v0[b]);
    float w0 = m.ball_w0[b];
    if (lane == 0) {
      x[n + b] = v0.f2();
      x[n + nb + b] = make_float2(w0, 0.0f);
      bvec[n + b] = (m.b_m * v0).f2();
      bvec[n + nb + b] = make_float2(m.b_I * w0, 0.0f);
    }
    float dl = m.b_m, da = m.b_I, unused = 0.0f;
    const uint32_t g0 = m.g_off[b], ng = m.g_off[b + 1] - g0;
    const uint32_t lq0 = m.lo_start[b], nlo = m.lo_start[b + 1] - lq0;
    const uint32_t l0 = m.l_off[b], nown = m.l_off[b + 1] - l0;
    const uint32_t cnt = ng + nlo + nown;
    for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
      const uint32_t e = c0 + lane;
      float tl = -0.0f, ta = -0.0f;
      if (e < ng) {
        tl = dt * mass * m.g_c[g0 + e];
        ta = dt * mass * m.g_l2[g0 + e];
      } else if (e < ng + nlo) {
        tl = dt * m.l_c[m.lo_list[lq0 + (e - ng)]];
      } else if (e < cnt) {
        tl = dt * m.l_c[l0 + (e - ng - nlo)];
      }
      lane_seq_sum3(dl, da, unused, tl, ta, -0.0f, min(32u, cnt - c0));
    }
    if (lane == 0) {
      diag[n + b] = dl;
      diag[n + nb + b] = da;
    }
  }
}

// ---------------------------------------------------------------- per-ball loops of the stages
// Each runs for the balls w0, w0 + nw, ... (w0: the calling warp's index over all of the mill's
// blocks, nw: their warp count), one warp per ball with no state shared between balls, so the
// mill's block and its helper blocks (mill_wide.cuh) can split them.

// Step 3.6b adhesion per ball (pbf.rs:1540-1602): candidates of each boundary point in
// for_each_near order, 32 at a time, merged per fluid particle in first-seen order; the ball's
// impulse and its items' velocity changes (item_v) and count (item_n).
static __device__ void adhesion_balls(const MillDev& m, const StepUniform& U, const GridHdr& hA, uint32_t w0, uint32_t nw) {
  const uint32_t nb = m.nb, count_pb = U.boundary_count;
  const float h = m.f_h, rho0 = m.f_rho0, mass = m.f_mass, dt = U.dt;
  const float2* X = m.fx;
  uint32_t* err = m.err;
  const float wett = clamp_r(U.slurry.wettability, 0.0f, 1.0f);
  const float h_adh = fmin_r(h, 2.0f * m.b_r);
  const float adhesion_accel = wett * 2.0f * fabsf(GRAVITY);
  const float range2 = h_adh * h_adh * (1.0f + 1e-4f);
  const float inner2 = 0.25f * h_adh * h_adh * (1.0f - 1e-4f);
  const uint32_t lane = tid() & 31u;
  uint32_t* slot = m.slot + (size_t)w0 * m.cap_nf;
  for (uint32_t b = w0; b < nb; b += nw) {
    const uint32_t base = b * m.cap_items;
    const MergeList L{m.item_j + base, m.item_w + base, m.item_v + base, nullptr, m.cap_items};
    uint32_t cnt = 0;
    bool overflow = false;
    const V2 xb(m.bx[b]);
    if (xb.finite()) {
      warp_near_multi(
          hA, m.gA, count_pb, [&](uint32_t q) { return xb + U.boundary_offset[q]; },
          [&](uint32_t j, bool valid) { return valid ? V2(X[j]) : V2(); },
          [&](uint32_t j, uint32_t q, V2 xj, bool valid) {
            bool acc = false;
            float w = 0.0f;
            V2 dir;
            if (valid) {
              const V2 bp = xb + U.boundary_offset[q];
              V2 delta = bp - xj;
              float r2 = delta.len2();
              if (!(r2 >= range2 || r2 <= inner2)) {
                float r = sqrtf(r2);
                if (!(!finite_f(r) || r <= 0.5f * h_adh || r >= h_adh)) {
                  w = mass * adhesion_kernel(r, h_adh) / rho0;
                  if (w > 0.0f) { acc = true; dir = w * (delta / r); }
                }
              }
            }
            warp_merge(acc, j, w, dir, 0.0f, slot, L, cnt, overflow);
          });
    }
    for (uint32_t s = lane; s < min(cnt, m.cap_items); s += 32) slot[L.j[s]] = NONE;
    __syncwarp();
    if (__any_sync(FULL, overflow)) { if (lane == 0) atomicOr(err, ERR_ITEMS); cnt = 0; }
    uint32_t used = 0;
    if (cnt > 0) {
      // dir_sum and weight_sum in item order (pbf.rs:1586-1594)
      float weight_sum = 0.0f, dsx = 0.0f, dsy = 0.0f;
      for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
        const uint32_t s = c0 + lane, lim = min(32u, cnt - c0);
        float ww = 0.0f;
        V2 dd;
        if (s < cnt) { ww = L.v0[s]; dd = V2(L.v1[s]); }
#pragma unroll
        for (uint32_t t = 0; t < 32; ++t) {
          const float xt = __shfl_sync(FULL, dd.x, t), yt = __shfl_sync(FULL, dd.y, t);
          const float wt = __shfl_sync(FULL, ww, t);
          if (t < lim) {
            dsx += xt;
            dsy += yt;
            weight_sum += wt;
          }
        }
      }
      V2 dir_sum(dsx, dsy);
      float pull_len = dir_sum.len();
      if (weight_sum > 1e-9f && pull_len > 1e-9f) {
        V2 ball_pull_dir = -dir_sum / pull_len;
        float coverage = fmin_r(weight_sum, 1.0f);
        float m_contrib = mass * weight_sum;
        float attach = m_contrib / (m.b_m + m_contrib);
        V2 dv_b = ball_pull_dir * (adhesion_accel * coverage * dt * attach);
        if (lane == 0) {
          m.imp[b] = (V2(m.imp[b]) + m.b_m * dv_b).f2();
          V2 lever = ball_pull_dir * m.b_r;
          m.ang[b] += m.b_m * cross2(lever, dv_b);
        }
        for (uint32_t s = lane; s < cnt; s += 32) {
          float frac = L.v0[s] / weight_sum;
          V2 dv_i = -(m.b_m * frac / mass) * dv_b;
          L.v1[s] = dv_i.f2();
        }
        used = cnt;
      }
    }
    if (lane == 0) m.item_n[b] = used;
    __syncwarp();
  }
}

// Per-ball item lists (cap_items per ball): fluid index, offset / lever, weight, second weight.
struct ItemLists {
  uint32_t* j;
  float2* v;
  float* w;
  float* w2;
};
__device__ __forceinline__ ItemLists mill_items(const MillDev& m) { return {m.item_j, m.item_v, m.item_w, m.item_w2}; }

// Boundary groups per ball (pbf.rs:2159-2232) on the fresh h-grid: candidates of each boundary
// point merged per fluid particle in first-seen order into the lists I; the ball's group count in
// g_off[b]. slot_warp: the warp's merge slot map (a warp index of the mill's blocks).
static __device__ void group_balls(const MillDev& m, const StepUniform& U, const GridHdr& hB, uint32_t w0, uint32_t nw,
                                   const ItemLists& I, uint32_t slot_warp) {
  const uint32_t nb = m.nb, count_pb = U.boundary_count;
  const float h = m.f_h;
  const float2* X = m.fx;
  uint32_t* err = m.err;
  const float eta2 = VISC_ETA * h * h;
  const float spiky_norm = -30.0f / (PI_F * powi5(h));
  const float range2 = h * h * (1.0f + 1e-4f);
  uint32_t* slot = m.slot + (size_t)slot_warp * m.cap_nf;
  for (uint32_t b = w0; b < nb; b += nw) {
    const uint32_t lane = tid() & 31u, base = b * m.cap_items;
    const MergeList L{I.j + base, I.w + base, I.v + base, I.w2 + base, m.cap_items};
    uint32_t cnt = 0;
    bool overflow = false;
    const V2 xb(m.bx[b]);
    if (xb.finite()) {
      struct XF {
        V2 x;
        float f;
      };
      warp_near_multi(
          hB, m.gB, count_pb, [&](uint32_t q) { return xb + U.boundary_offset[q]; },
          [&](uint32_t j, bool valid) {
            XF d{V2(), 0.0f};
            if (valid) {
              d.x = V2(X[j]);
              d.f = m.f_tmp[j];
            }
            return d;
          },
          [&](uint32_t j, uint32_t q, XF d, bool valid) {
            bool acc = false;
            float c = 0.0f, lever2_c = 0.0f;
            V2 lever_c;
            if (valid) {
              const V2 bp = xb + U.boundary_offset[q];
              V2 delta = d.x - bp;
              float r2 = delta.len2();
              if (!(r2 >= range2)) {
                float r = sqrtf(r2);
                if (!(!finite_f(r) || r >= h || r <= 1e-9f)) {
                  float dot_abs = fabsf(spiky_norm * (h - r) * (h - r) * r);
                  c = d.f * dot_abs / (r2 + eta2);
                  if (c > 0.0f) {
                    acc = true;
                    V2 lever = bp - xb;
                    lever_c = c * lever;
                    lever2_c = c * lever.len2();
                  }
                }
              }
            }
            warp_merge(acc, j, c, lever_c, lever2_c, slot, L, cnt, overflow);
          });
    }
    for (uint32_t s = lane; s < min(cnt, m.cap_items); s += 32) slot[L.j[s]] = NONE;
    __syncwarp();
    if (__any_sync(FULL, overflow)) { if (lane == 0) atomicOr(err, ERR_ITEMS); cnt = 0; }
    if (lane == 0) m.g_off[b] = cnt;
    __syncwarp();
  }
}

// Squeeze links per ball (pbf.rs:544-625): candidates j > i in for_each_near order, ordered
// compaction, then the wall link, each film evaluated once; ball i's links go to its slots
// [i K, i K + K) of the record scratch and its count to l_off[i]. Returns the thread's part of
// the count of links in range.
static __device__ uint32_t link_balls(const MillDev& m, const StepUniform& U, const GridHdr& hBall, uint32_t w0, uint32_t nw) {
  const uint32_t nb = m.nb;
  const float h = m.f_h, dt = U.dt;
  uint32_t* err = m.err;
  const float r = m.b_r;
  const double dxd = (double)(0.5f * h);
  const float reach = (float)(8.0 * dxd);
  const float c_max = 8.0f * m.b_m / fmax_r(dt, 1e-12f);
  const float range2 = (2.0f * r + reach) * (2.0f * r + reach) * (1.0f + 1e-4f);
  const uint32_t K = min(nb + 1u, 512u);
  uint32_t in_range = 0;
  for (uint32_t i = w0; i < nb; i += nw) {
    const uint32_t lane = tid() & 31u;
    const V2 xi(m.bx[i]), v0i(m.ball_v0[i]);
    const uint32_t base = i * K;
    uint32_t c = 0, inr = 0;
    if (xi.finite()) {
      struct XV {
        V2 x, v0;
      };
      warp_near_multi(
          hBall, m.gBall, 1u, [&](uint32_t) { return xi; },
          [&](uint32_t j, bool valid) {
            XV d{V2(), V2()};
            if (valid && j > i) {
              d.x = V2(m.bx[j]);
              d.v0 = V2(m.ball_v0[j]);
            }
            return d;
          },
          [&](uint32_t j, uint32_t, XV d, bool valid) {
            const bool cand = valid && j > i;
            LinkEval L{false, false, V2(), 0.0f};
            if (cand) L = link_pair(m, U, xi, v0i, d.x, d.v0, reach, range2, dxd, c_max, true);
            inr += __popc(__ballot_sync(FULL, cand && L.in_range));
            const uint32_t bal = __ballot_sync(FULL, cand && L.emit);
            const uint32_t q = c + __popc(bal & ((1u << lane) - 1u));
            if (cand && L.emit && q < K) {
              m.rec_i[base + q] = j;
              m.rec_J[base + q] = L.n.f2();
              m.rec_L[base + q] = L.c;
            }
            c += __popc(bal);
          });
      if (lane == 0) {
        LinkEval W = link_wall(m, U, i, reach, dxd, c_max);
        if (W.in_range) inr += 1;
        if (W.emit) {
          if (c < K) { m.rec_i[base + c] = NONE; m.rec_J[base + c] = W.n.f2(); m.rec_L[base + c] = W.c; }
          ++c;
        }
      }
    }
    if (lane == 0) {
      if (c > K) { atomicOr(err, ERR_LINKS); c = K; }
      m.l_off[i] = c;
      in_range += inr;
    }
    __syncwarp();
  }
  return in_range;
}

// Squeeze-link candidates per ball (the geometry of link_balls, before the velocity test): for
// the balls w0, w0 + nw, ..., the partners j > i in for_each_near order that are within reach, with
// the normal and film coefficient link_pair gives them, into lk_* (count lk_cnt[i]; a ball with
// more candidates than its K slots counts into *over and is left for the full path), and the wall
// candidate in lk_winr / lk_wn / lk_wc. link_pair and link_wall evaluate the same expressions;
// only the test n . (v0_i - v0_j) > 0 (n . v0_i > 0 for the wall) is left to links_from_candidates.
static __device__ void link_candidate_balls(const MillDev& m, const StepUniform& U, const GridHdr& hBall, uint32_t w0,
                                            uint32_t nw, uint32_t* over) {
  const uint32_t nb = m.nb;
  const float h = m.f_h, dt = U.dt;
  const float r = m.b_r;
  const double dxd = (double)(0.5f * h);
  const float reach = (float)(8.0 * dxd);
  const float c_max = 8.0f * m.b_m / fmax_r(dt, 1e-12f);
  const float range2 = (2.0f * r + reach) * (2.0f * r + reach) * (1.0f + 1e-4f);
  const uint32_t K = min(nb + 1u, 512u);
  for (uint32_t i = w0; i < nb; i += nw) {
    const uint32_t lane = tid() & 31u;
    const V2 xi(m.bx[i]);
    const uint32_t base = i * K;
    uint32_t c = 0;
    if (xi.finite()) {
      warp_near_multi(
          hBall, m.gBall, 1u, [&](uint32_t) { return xi; },
          [&](uint32_t j, bool valid) { return valid && j > i ? V2(m.bx[j]) : V2(); },
          [&](uint32_t j, uint32_t, V2 xj, bool valid) {
            bool keep = false;
            V2 nrm;
            float cf = 0.0f;
            if (valid && j > i) {
              V2 e = xj - xi;
              if (!(e.len2() >= range2 || !e.finite())) {
                float dist = e.len();
                float gap = dist - 2.0f * r;
                if (!(gap >= reach || dist < 1e-9f)) {
                  keep = true;
                  nrm = e / dist;
                  double weight = 1.0 - resolved_ratio((double)gap / dxd);
                  double hh = (double)gap > 0.02 * (double)r ? (double)gap : 0.02 * (double)r;
                  double cc = weight * film_coefficient(U.pair_film, hh);
                  cf = fmin_r(1.0f * (float)cc, c_max);
                }
              }
            }
            const uint32_t bal = __ballot_sync(FULL, keep);
            const uint32_t q = c + __popc(bal & ((1u << lane) - 1u));
            if (keep && q < K) {
              m.lk_j[base + q] = j;
              m.lk_n[base + q] = nrm.f2();
              m.lk_c[base + q] = cf;
            }
            c += __popc(bal);
          });
    }
    if (lane == 0) {
      uint32_t winr = 0;
      V2 wn;
      float wc = 0.0f;
      const float dist = xi.len();
      const float gap = U.drum_radius - r - dist;
      if (gap < reach && dist > 1e-9f) {
        winr = 1u;
        wn = xi / dist;
        double weight = 1.0 - resolved_ratio((double)gap / dxd);
        double hh = (double)gap > 0.02 * (double)r ? (double)gap : 0.02 * (double)r;
        double cc = weight * film_coefficient(U.wall_film, hh);
        wc = fmin_r(1.0f * (float)cc, c_max);
      }
      m.lk_winr[i] = winr;
      m.lk_wn[i] = wn.f2();
      m.lk_wc[i] = wc;
      if (c > K) { atomicAdd(over, 1u); c = K; }
      m.lk_cnt[i] = c;
    }
    __syncwarp();
  }
}

// Squeeze links per ball from the candidates link_candidate_balls listed, once ball_v0 is known:
// candidate j is a link when n . (v0_i - v0_j) > 0 (the wall when n . v0_i > 0), kept in candidate
// order, then the wall, into the record scratch slots [i K, i K + K) and the count into l_off[i]
// as link_balls leaves them. Returns the thread's part of the count of candidates in range.
static __device__ uint32_t links_from_candidates(const MillDev& m, uint32_t w0, uint32_t nw) {
  const uint32_t nb = m.nb;
  const uint32_t K = min(nb + 1u, 512u);
  uint32_t in_range = 0;
  for (uint32_t i = w0; i < nb; i += nw) {
    const uint32_t lane = tid() & 31u, base = i * K, cnt = m.lk_cnt[i];
    const V2 v0i(m.ball_v0[i]);
    uint32_t c = 0;
    for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
      const uint32_t q = c0 + lane;
      bool emit = false;
      uint32_t j = 0;
      V2 nrm;
      if (q < cnt) {
        j = m.lk_j[base + q];
        nrm = V2(m.lk_n[base + q]);
        emit = !(nrm.dot(v0i - V2(m.ball_v0[j])) <= 0.0f);
      }
      const uint32_t bal = __ballot_sync(FULL, emit);
      const uint32_t pos = c + __popc(bal & ((1u << lane) - 1u));
      if (emit && pos < K) {
        m.rec_i[base + pos] = j;
        m.rec_J[base + pos] = nrm.f2();
        m.rec_L[base + pos] = m.lk_c[base + q];
      }
      c += __popc(bal);
    }
    if (lane == 0) {
      const uint32_t winr = m.lk_winr[i];
      if (winr) {
        const V2 wn(m.lk_wn[i]);
        if (!(wn.dot(v0i) <= 0.0f)) {
          if (c < K) { m.rec_i[base + c] = NONE; m.rec_J[base + c] = wn.f2(); m.rec_L[base + c] = m.lk_wc[i]; }
          ++c;
        }
      }
      if (c > K) { atomicOr(m.err, ERR_LINKS); c = K; }
      m.l_off[i] = c;
      in_range += cnt + winr;
    }
    __syncwarp();
  }
  return in_range;
}

// Drag item lists per ball (pbf.rs:1794-1822): fluid particles within r + h of the ball centre in
// for_each_near order, with their offsets and weights (item_j / item_v / item_w, count item_n).
// Returns the thread's part of the item count.
static __device__ uint32_t drag_item_balls(const MillDev& m, const GridHdr& hB, uint32_t w0, uint32_t nw) {
  const uint32_t nb = m.nb;
  const float h = m.f_h;
  const float2* X = m.fx;
  uint32_t* err = m.err;
  const float h_c = m.b_r + h;
  const float w_hc0 = fmax_r(poly6(0.0f, h_c), 1e-12f);
  uint32_t items = 0;
  for (uint32_t b = w0; b < nb; b += nw) {
    const uint32_t lane = tid() & 31u, base = b * m.cap_items;
    uint32_t cnt = 0;
    const V2 xb(m.bx[b]);
    if (xb.finite()) {
      warp_near_multi(
          hB, m.gB, 1u, [&](uint32_t) { return xb; },
          [&](uint32_t j, bool valid) { return valid ? V2(X[j]) : V2(); },
          [&](uint32_t j, uint32_t, V2 xj, bool valid) {
        bool keep = false;
        V2 r_i;
        float phi = 0.0f;
        if (valid) {
          r_i = xj - xb;
          float r2 = r_i.len2();
          if (!(!finite_f(r2) || r2 >= h_c * h_c)) {
            phi = poly6(r2, h_c) / w_hc0;
            keep = phi > 0.0f;
          }
        }
        const uint32_t bal = __ballot_sync(FULL, keep);
        const uint32_t pos = cnt + __popc(bal & ((1u << lane) - 1u));
        if (keep && pos < m.cap_items) {
          m.item_j[base + pos] = j;
          m.item_v[base + pos] = r_i.f2();
          m.item_w[base + pos] = phi;
        }
        cnt += __popc(bal);
      });
    }
    if (cnt > m.cap_items) { if (lane == 0) atomicOr(err, ERR_ITEMS); cnt = 0; }
    if (lane == 0) { m.item_n[b] = cnt; items += cnt; }
    __syncwarp();
  }
  return items;
}

// Buoyancy item lists per ball (pbf.rs:2042-2060) on the stale step-2 grid: fluid particles with a
// positive poly6 weight in for_each_near order, their weights, and the local density (item_v[0]).
// Returns the thread's part of the item count.
static __device__ uint32_t buoyancy_item_balls(const MillDev& m, const GridHdr& hA, uint32_t w0, uint32_t nw,
                                               const ItemLists& I, uint32_t* item_n) {
  const uint32_t nb = m.nb;
  const float h = m.f_h, mass = m.f_mass;
  const float2* X = m.fx;
  uint32_t* err = m.err;
  uint32_t items = 0;
  for (uint32_t b = w0; b < nb; b += nw) {
    const uint32_t lane = tid() & 31u, base = b * m.cap_items;
    uint32_t cnt = 0;
    const V2 xb(m.bx[b]);
    float rho_local = 0.0f;
    if (xb.finite()) {
      warp_near_multi(
          hA, m.gA, 1u, [&](uint32_t) { return xb; },
          [&](uint32_t j, bool valid) { return valid ? V2(X[j]) : V2(); },
          [&](uint32_t j, uint32_t, V2 xj, bool valid) {
        float w = 0.0f;
        if (valid) w = mass * poly6((xb - xj).len2(), h);
        const bool keep = w > 0.0f;
        const uint32_t bal = __ballot_sync(FULL, keep);
        const uint32_t pos = cnt + __popc(bal & ((1u << lane) - 1u));
        if (keep && pos < m.cap_items) { I.j[base + pos] = j; I.w[base + pos] = w; }
#pragma unroll
        for (int t = 0; t < 32; ++t) {
          const float wt = __shfl_sync(FULL, w, t);
          if ((bal >> t) & 1u) rho_local += wt;
        }
        cnt += __popc(bal);
      });
    }
    if (cnt > m.cap_items) { if (lane == 0) atomicOr(err, ERR_ITEMS); cnt = 0; }
    if (lane == 0) {
      item_n[b] = rho_local > 0.0f ? cnt : 0u;
      if (rho_local > 0.0f) items += cnt;
      I.v[base] = make_float2(rho_local, 0.0f);
    }
    __syncwarp();
  }
  return items;
}

// The drag sweep's per-ball quantities that read only the item geometry (pbf.rs:1845-1905), for
// the balls w0, w0 + nw, ...: entrained mass and inertia, centroid and the s-gate sums, summed in
// item order; written to drag_pre[8 b ..] (mass, inertia, centroid x, y, s_acc, s_scale).
static __device__ void drag_pre_balls(const MillDev& m, uint32_t w0, uint32_t nw) {
  const uint32_t nb = m.nb, lane = tid() & 31u;
  const float mass = m.f_mass;
  for (uint32_t b = w0; b < nb; b += nw) {
    const uint32_t cnt = m.item_n[b], base = b * m.cap_items;
    float m_ent = 0.0f, i_ent = 0.0f, rsx = 0.0f, rsy = 0.0f;
    for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
      const uint32_t s = c0 + lane, lim = min(32u, cnt - c0);
      float w = 0.0f, r2w = 0.0f;
      V2 rw;
      if (s < cnt) {
        V2 r_i(m.item_v[base + s]);
        w = mass * m.item_w[base + s];
        rw = w * r_i;
        r2w = w * r_i.len2();
      }
#pragma unroll
      for (uint32_t t = 0; t < 32; ++t) {
        const float wt = __shfl_sync(FULL, w, t), xt = __shfl_sync(FULL, rw.x, t);
        const float yt = __shfl_sync(FULL, rw.y, t), it = __shfl_sync(FULL, r2w, t);
        if (t < lim) {
          m_ent += wt;
          rsx += xt;
          rsy += yt;
          i_ent += it;
        }
      }
    }
    V2 r_bar;
    float s_acc = 0.0f, s_scale = 0.0f;
    if (cnt > 0 && !(m_ent <= 1e-12f)) {
      r_bar = V2(rsx, rsy) / m_ent;
      if (i_ent > 1e-12f) {
        const V2 p_bar(-r_bar.y, r_bar.x);
        for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
          const uint32_t s = c0 + lane, lim = min(32u, cnt - c0);
          float sv = 0.0f, ss = 0.0f;
          if (s < cnt) {
            V2 r_i(m.item_v[base + s]);
            float phi = m.item_w[base + s];
            V2 perp_i(-r_i.y, r_i.x);
            float phi2 = phi * phi;
            sv = mass * phi2 * cross2(r_i, perp_i - p_bar);
            ss = mass * phi2 * r_i.len2();
          }
#pragma unroll
          for (uint32_t t = 0; t < 32; ++t) {
            const float at = __shfl_sync(FULL, sv, t), st = __shfl_sync(FULL, ss, t);
            if (t < lim) {
              s_acc += at;
              s_scale += st;
            }
          }
        }
      }
    }
    if (lane == 0) {
      float* P = m.drag_pre + 8u * b;
      P[0] = m_ent;
      P[1] = i_ent;
      P[2] = r_bar.x;
      P[3] = r_bar.y;
      P[4] = s_acc;
      P[5] = s_scale;
    }
  }
}

// The per-ball sweeps' slot for the ball a warp is running (one per warp; indices DS_* for the drag
// sweep, BS_* for the buoyancy sweep) and the running sweep's constants (DK_* / BK_*), in shared
// memory so that the per-ball bodies keep few values in registers across the dependency wait.
enum : uint32_t {
  DS_M_ENT = 0, DS_I_ENT = 1, DS_R_BAR = 2, DS_S_ACC = 4, DS_S_SCALE = 5, DS_PRE = 6,  // drag_pre[0..5]
  DS_VB = 6, DS_OMB = 8, DS_DV_B = 9, DS_DW_B = 11, DS_LIN_DEN = 12, DS_ROT_DEN = 13, DS_NEG_BM_MENT = 14,
  DS_SLOT = 15
};
enum : uint32_t { BS_RHO_LOCAL = 0, BS_DEN = 1, BS_XB = 2, BS_IMPULSE = 4 };
enum : uint32_t {
  DK_MASS, DK_RHO0, DK_MASS_TRUE, DK_BETA, DK_DT, DK_I_B, DK_H_C, DK_ROT_CAP, DK_B_M, DK_B_RTRUE, DK_FORM, DK_CAP
};
enum : uint32_t { BK_RHO0, BK_OM_ABS, BK_AREA, BK_DT, BK_MASS };
constexpr uint32_t SWEEP_CONSTS = 12;  // DK_* and BK_* indices are below it
constexpr uint32_t DRAG_LIVE = 0x80000000u;
__shared__ float g_ball_slot[MAX_BLOCK_WARPS][DS_SLOT];
__shared__ float g_sweep_const[SWEEP_CONSTS];

// The drag sweep proper (pbf.rs:1824-2011): balls in dependency order over the item lists, on the
// velocities V; the constants are in g_sweep_const. Its own function, so that the per-ball bodies
// are register-allocated apart from the set-up around them.
static __device__ __noinline__ void drag_sweep(const MillDev& m, const StepUniform& U, StepOut& out, uint32_t* err,
                                               float2* V, uint32_t* done, const uint32_t* order) {
  const uint32_t nb = m.nb;
  const bool want_mom = U.want_momentum != 0;
  // Lane l holds item l of the ball (items from 32 on are read from the lists when needed); the
  // ball's own quantities sit in its warp's slot (g_ball_slot) from the prefetch to the post.
  struct DragBall {
    uint32_t cnt;  // item count, DRAG_LIVE set when the ball takes part (entrained mass > 1e-12)
    uint32_t j;
    V2 r_i;
    float phi;
    V2 dv_i;
  };
  ball_dataflow(
      nb, m.rec_off, m.rec_pred, done, order, U.sweep_warps, U.spin_ns, U.spin_limit, U.skip_done_ball, err,
      &out.stage[32],
      // before the wait: the item data and the geometry-only quantities computed for every ball
      // ahead of the sweep (drag_pre_balls)
      [&](uint32_t b, int lane) {
        DragBall q;
        q.cnt = m.item_n[b];
        q.j = 0;
        q.phi = 0.0f;
        if (q.cnt == 0) return q;
        const uint32_t base = b * m.cap_items;
        if ((uint32_t)lane < q.cnt) {
          q.j = m.item_j[base + lane];
          q.r_i = V2(m.item_v[base + lane]);
          q.phi = m.item_w[base + lane];
        }
        // slot: entrained mass, inertia, centroid x, y, s_acc, s_scale (drag_pre), the ball's
        // velocity x, y and spin
        float* sl = g_ball_slot[threadIdx.x >> 5];
        __syncwarp();  // the previous ball's post has read the slot
        if (lane < DS_PRE) sl[lane] = m.drag_pre[8u * b + lane];
        else if (lane < DS_OMB) sl[lane] = reinterpret_cast<const float*>(m.bv + b)[lane - DS_VB];
        else if (lane == DS_OMB) sl[lane] = m.bom[b];
        // the relaxation's terms that do not read the swept velocities (the same operations as on
        // the chain, done ahead): b_m + m_ent, i_b + i_ent, -(b_m / m_ent)
        else if (lane == DS_LIN_DEN) sl[lane] = g_sweep_const[DK_B_M] + m.drag_pre[8u * b + DS_M_ENT];
        else if (lane == DS_ROT_DEN) sl[lane] = g_sweep_const[DK_I_B] + m.drag_pre[8u * b + DS_I_ENT];
        else if (lane == DS_NEG_BM_MENT) sl[lane] = -(g_sweep_const[DK_B_M] / m.drag_pre[8u * b + DS_M_ENT]);
        if (!(m.drag_pre[8u * b] <= 1e-12f)) q.cnt |= DRAG_LIVE;  // (a NaN mass takes part too)
        return q;
      },
      // on the chain: entrained velocity and angular momentum, the relaxation, the fluid updates
      [&](uint32_t b, int lane, DragBall& q) {
        if (!(q.cnt & DRAG_LIVE)) return;
        const uint32_t base = b * m.cap_items, cnt = q.cnt & ~DRAG_LIVE;
        const float* sl = g_ball_slot[threadIdx.x >> 5];
        const float* K = g_sweep_const;
        float2* const Vl = V;
        const float mass_l = K[DK_MASS];
        float l_sum = 0.0f, vsx = 0.0f, vsy = 0.0f;
        for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
          const uint32_t s = c0 + lane, lim = min(32u, cnt - c0);
          float lw = 0.0f;
          V2 vw;
          if (s < cnt) {
            const V2 r_i = s < 32 ? q.r_i : V2(m.item_v[base + s]);
            const V2 vj(Vl[s < 32 ? q.j : m.item_j[base + s]]);
            const float w = mass_l * (s < 32 ? q.phi : m.item_w[base + s]);
            vw = w * vj;
            lw = w * cross2(r_i, vj);
          }
          lane_seq_sum3(vsx, vsy, l_sum, vw.x, vw.y, lw, lim);
        }
        const float m_ent = sl[DS_M_ENT], i_ent = sl[DS_I_ENT], i_b = K[DK_I_B];
        V2 v_bar = V2(vsx, vsy) / m_ent;
        V2 v_rel = v_bar - V2(sl[DS_VB], sl[DS_VB + 1]);
        float speed_rel = v_rel.len();
        const float rho0_l = K[DK_RHO0];
        // (K[DK_FORM] = 0.5 rho0 1 (2 r_true), the left part of the product, formed ahead)
        float inv_tau_form = (speed_rel > 1e-6f && rho0_l > 0.0f) ? K[DK_FORM] * speed_rel / K[DK_MASS_TRUE] : 0.0f;
        float bt = K[DK_BETA] * (1.0f - expf_r(-K[DK_DT] * (0.0f + inv_tau_form)));
        float a_lin = bt * m_ent / sl[DS_LIN_DEN];
        V2 dv_b = a_lin * v_rel;
        float dw_b = 0.0f, c_rot = 0.0f;
        if (i_ent > 1e-12f) {
          float omega_bar = l_sum / i_ent;
          float a_rot = bt * i_ent / sl[DS_ROT_DEN];
          float candidate_dw = a_rot * (omega_bar - sl[DS_OMB]);
          const float s_acc = sl[DS_S_ACC];
          if (fabsf(s_acc) > 0.1f * sl[DS_S_SCALE]) {
            float raw_c_rot = -i_b * candidate_dw / s_acc;
            const float cap = K[DK_CAP];  // rot_cap / (2 h_c), formed ahead
            c_rot = clamp_r(raw_c_rot, -cap, cap);
            dw_b = -c_rot * s_acc / i_b;
          }
        }
        const V2 p_bar(-sl[DS_R_BAR + 1], sl[DS_R_BAR]);  // read only when c_rot != 0 (i_ent > 1e-12)
        for (uint32_t s = lane; s < cnt; s += 32) {
          const uint32_t j = s < 32 ? q.j : m.item_j[base + s];
          const V2 r_i = s < 32 ? q.r_i : V2(m.item_v[base + s]);
          const float phi = s < 32 ? q.phi : m.item_w[base + s];
          V2 dv_i = sl[DS_NEG_BM_MENT] * dv_b * phi;  // -(b_m / m_ent), formed ahead
          if (c_rot != 0.0f) {
            V2 perp_i(-r_i.y, r_i.x);
            dv_i += c_rot * phi * (perp_i - p_bar);
          }
          Vl[j] = (V2(Vl[j]) + dv_i).f2();
          if (s < 32) q.dv_i = dv_i;
          else if (want_mom) m.rec_M[m.rec_off[b] + s] = (mass_l * dv_i).f2();
        }
        if (lane == 0) {
          float* slw = g_ball_slot[threadIdx.x >> 5];
          slw[DS_DV_B] = dv_b.x;
          slw[DS_DV_B + 1] = dv_b.y;
          slw[DS_DW_B] = dw_b;
        }
      },
      // after the flag: the ball's impulse and angular impulse, the momentum records
      [&](uint32_t b, int lane, DragBall& q) {
        if (!(q.cnt & DRAG_LIVE)) return;
        const uint32_t cnt = q.cnt & ~DRAG_LIVE;
        if (want_mom && (uint32_t)lane < cnt) m.rec_M[m.rec_off[b] + lane] = (m.f_mass * q.dv_i).f2();
        if (lane == 0) {
          const float* sl = g_ball_slot[threadIdx.x >> 5];
          const V2 dv_b(sl[DS_DV_B], sl[DS_DV_B + 1]), r_bar(sl[DS_R_BAR], sl[DS_R_BAR + 1]);
          m.imp[b] = (V2(m.imp[b]) + m.b_m * dv_b).f2();
          m.ang[b] += m.b_I * sl[DS_DW_B] + m.b_m * cross2(r_bar, dv_b);
          m.item_n[b] = cnt | 0x80000000u;  // mark: contributed fluid momentum records
        }
      });
}

// Step 6.5 (pbf.rs:1777-2013): the drag sweep on the velocities V (positions X), in its own
// function so that the sweep's per-ball state gets the whole register budget. Returns false when
// the item lists failed (the error is in *err).
static __device__ __noinline__ bool drag_step(const MillDev& m, const StepUniform& U, StepOut& out, uint32_t* err,
                                              FluidShared& S, float2* X, float2* V, uint32_t* done,
                                              uint32_t* scratch, uint32_t scratch_words,
                                              const uint32_t** order_out, uint32_t* beside_out, bool listed) {
  const uint32_t n = m.nf, nb = m.nb;
  const float h = m.f_h, rho0 = m.f_rho0, mass = m.f_mass, dt = U.dt;
  (void)rho0;
  const float mu = fmax_r(U.slurry.viscosity_pa_s, 0.0f);
  if (nb > 0 && m.b_r > 0.0f && m.b_rtrue > 0.0f && mu > 1e-6f) {
    const float beta_b = clamp_r(U.slurry.ball_no_slip, 0.0f, 1.0f);
    const float rot_cap = 0.2f * fluid_vmax(U);
    const float rho_ball = m.b_m / (PI_F * m.b_r * m.b_r);
    const float mass_true = rho_ball * PI_F * m.b_rtrue * m.b_rtrue;
    if (beta_b > 0.0f) {
      const float h_c = m.b_r + h;
      const uint32_t* order = nullptr;
      if (listed) {
        // the helper blocks listed the items, records, claim order and pre-sums during steps 5-6
        // (WIDE_DRAG_LISTS); the claim order lives in d_order, not in this block's scratch, so
        // the buoyancy sweep does not reuse it
        wide_finish(m);
        const uint32_t n_items = wide_counter(m);
        if (tid() == 0) out.ctr.n_coupling_items += n_items;
        __syncthreads();
        if (*err) return false;
        stage_mark(out.stage, 24);
        order = m.wide->drag_order_ok ? m.d_order : nullptr;
        stage_mark(out.stage, 25);
      } else {
        grid_build(X, n, fmax_r(h_c, 1e-6f), m.gB, S.hB, err);
        // item lists per ball in for_each_near order (positions do not change during the sweep):
        // one warp per ball, an ordered compaction of each 32-candidate chunk
        uint32_t n_items = 0;
        wide_phase(m, WIDE_DRAG_ITEMS, &S.hB,
                   [&](uint32_t w0, uint32_t nw) { n_items += drag_item_balls(m, S.hB, w0, nw); });
        n_items = block_sum_u(n_items) + wide_counter(m);
        if (tid() == 0) out.ctr.n_coupling_items += n_items;
        __syncthreads();
        if (*err) return false;
        stage_mark(out.stage, 24);
        const uint32_t nrec = pack_ball_items(m.item_j, m.item_n, m.cap_items, nb, m.rec_off, m.rec_i, m.rec_b);
        LevelScratch L;
        const bool by_level = U.sweep_order == 0 && level_scratch(nb, scratch, scratch_words, L);
        ball_item_preds(m.rec_i, m.rec_b, nrec, n, nb, m.bk_start, m.bk_cur, m.bk_order, m.rec_pred,
                        by_level ? &L : nullptr);
        order = by_level ? ball_level_order(nb, m.rec_off, m.rec_pred, L) : nullptr;
        *order_out = order;
        stage_mark(out.stage, 25);
        wide_phase(m, WIDE_DRAG_PRE, nullptr, [&](uint32_t w0, uint32_t nw) { drag_pre_balls(m, w0, nw); });
      }
      // the sweep's constants, read from shared memory by the per-ball bodies
      if (tid() == 0) {
        float* K = g_sweep_const;
        K[DK_MASS] = mass;
        K[DK_RHO0] = rho0;
        K[DK_MASS_TRUE] = mass_true;
        K[DK_BETA] = beta_b;
        K[DK_DT] = dt;
        K[DK_I_B] = m.b_I;
        K[DK_H_C] = h_c;
        K[DK_ROT_CAP] = rot_cap;
        K[DK_B_M] = m.b_m;
        K[DK_B_RTRUE] = m.b_rtrue;
        K[DK_FORM] = 0.5f * rho0 * 1.0f * (2.0f * m.b_rtrue);
        const float max_lever = 2.0f * h_c;
        K[DK_CAP] = max_lever > 1e-9f ? rot_cap / max_lever : 0.0f;
      }
      __syncthreads();
      // With two or more helper blocks, the helpers do what reads only the final positions beside
      // the sweep (beside_drag): the buoyancy item lists, records and claim order and, without the
      // Bingham rheology (its viscosity reads the velocities), the density recompute, the
      // viscosity's Morris weights and its boundary groups.
      if (m.helpers >= 2 && m.bi_j != nullptr) {
        const bool bingham = U.slurry.rheology == MG_RHEOLOGY_BINGHAM && U.slurry.yield_stress_pa > 0.0f;
        const uint32_t tasks = BESIDE_BUOY | (bingham ? 0u : BESIDE_VISC);
        wide_publish(m, WIDE_BESIDE_DRAG, &S.hA, nullptr, nullptr, [&](WideCtl* c) {
          c->beside_tasks = tasks;
          c->beside_mu = mu;
          c->beside_grid_seq = 0u;
          c->beside_buoy_blocks = 0u;
          c->beside_nrec = 0u;
          c->beside_order_ok = 0u;
          c->beside_link_over = 0u;
          c->beside_group_blocks = 0u;
          c->beside_ngroups = 0u;
          c->beside_groups_ok = 0u;
        });
        *beside_out = tasks;
      }
      drag_sweep(m, U, out, err, V, done, order);
      if (tid() == 0 && U.want_momentum) {
        V2 mom(S.fscal[0], S.fscal[1]);
        for (uint32_t b = 0; b < nb; ++b) {
          if (!(m.item_n[b] & 0x80000000u)) continue;
          for (uint32_t r = m.rec_off[b]; r < m.rec_off[b + 1]; ++r) mom += V2(m.rec_M[r]);
        }
        S.fscal[0] = mom.x;
        S.fscal[1] = mom.y;
      }
      __syncthreads();
      stage_mark(out.stage, 26);
    }
  }
  return true;
}

// The buoyancy sweep's item lists and records: per-ball item counts, fluid indices, weights and
// local densities (v[b * cap_items].x), record offsets per ball and predecessor balls.
struct BuoyLists {
  const uint32_t* n;
  const uint32_t* j;
  const float* w;
  const float2* v;
  const uint32_t* rec_off;
  const uint32_t* rec_pred;
};

// The buoyancy sweep proper (pbf.rs:2042-2121): balls in dependency order over the item lists BL,
// on the velocities V at positions X. Its own function, like drag_sweep.
static __device__ __noinline__ void buoyancy_sweep(const MillDev& m, const StepUniform& U, StepOut& out,
                                                   uint32_t* err, const float2* X, float2* V, uint32_t* done,
                                                   const uint32_t* order, const BuoyLists& BL) {
  const uint32_t nb = m.nb;
  const bool want_mom = U.want_momentum != 0;
  if (tid() == 0) {
    float* K = g_sweep_const;
    K[BK_RHO0] = m.f_rho0;
    K[BK_OM_ABS] = fabsf(U.drum_omega);
    K[BK_AREA] = PI_F * m.b_r * m.b_r;
    K[BK_DT] = U.dt;
    K[BK_MASS] = m.f_mass;
  }
  __syncthreads();
  // Lane l holds item l of the ball (items from 32 on are read from the lists when needed); the
  // ball's local density, weight sum, position and impulse sit in its warp's slot.
  struct BuoyBall {
    uint32_t cnt, j;
    float w, frac, d2;
    V2 d, dv;
    bool valid;
  };
  ball_dataflow(
      nb, BL.rec_off, BL.rec_pred, done, order, U.sweep_warps, U.spin_ns, U.spin_limit, NONE, err, &out.stage[35],
      // before the wait: item geometry, the weight sum and the weight fractions, which the sweep does
      // not change
      [&](uint32_t b, int lane) {
        BuoyBall q;
        q.cnt = BL.n[b];
        q.j = 0;
        q.w = 0.0f;
        q.valid = false;
        if (q.cnt == 0) return q;
        const uint32_t base = b * m.cap_items, cnt = q.cnt;
        const float rho_local = BL.v[base].x;
        if ((uint32_t)lane < cnt) {
          q.j = BL.j[base + lane];
          q.w = BL.w[base + lane];
          q.d = V2(X[q.j]);
          q.d2 = q.d.len2();
          q.valid = !(q.d2 <= 1e-12f);
          q.frac = q.w / rho_local;
        }
        // the weight sum over the valid items in item order (an invalid item adds -0.0: no change)
        float den = 0.0f;
        for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
          const uint32_t s = c0 + lane, lim = min(32u, cnt - c0);
          float dvw = -0.0f;
          if (s < cnt) {
            if (s < 32) {
              if (q.valid) dvw = q.w;
            } else if (!(V2(X[BL.j[base + s]]).len2() <= 1e-12f)) {
              dvw = BL.w[base + s];
            }
          }
          lane_seq_sum1(den, dvw, lim);
        }
        float* sl = g_ball_slot[threadIdx.x >> 5];
        __syncwarp();  // the previous ball's post has read the slot
        if (lane == 0) {
          sl[BS_RHO_LOCAL] = rho_local;
          sl[BS_DEN] = den;
        } else if (lane <= 2) {
          sl[BS_XB + lane - 1] = reinterpret_cast<const float*>(m.bx + b)[lane - 1];
        }
        return q;
      },
      // on the chain: the local rotation rate from the current velocities, the fluid updates
      [&](uint32_t b, int lane, BuoyBall& q) {
        if (q.cnt == 0) return;
        const uint32_t base = b * m.cap_items, cnt = q.cnt;
        const float* sl = g_ball_slot[threadIdx.x >> 5];
        const float* K = g_sweep_const;
        float2* const V_l = V;
        // the rotation-rate numerator over the valid items in item order (invalid items add -0.0)
        float num = 0.0f;
        for (uint32_t c0 = 0; c0 < cnt; c0 += 32) {
          const uint32_t s = c0 + lane, lim = min(32u, cnt - c0);
          float nv = -0.0f;
          if (s < cnt) {
            if (s < 32) {
              if (q.valid) nv = q.w * cross2(q.d, V2(V_l[q.j])) / q.d2;
            } else {
              uint32_t j = BL.j[base + s];
              V2 d(X[j]);
              float d2 = d.len2();
              if (!(d2 <= 1e-12f)) nv = BL.w[base + s] * cross2(d, V2(V_l[j])) / d2;
            }
          }
          lane_seq_sum1(num, nv, lim);
        }
        const float rho_local = sl[BS_RHO_LOCAL], den = sl[BS_DEN], om_abs = K[BK_OM_ABS];
        const float rho_eff = fmin_r(rho_local, K[BK_RHO0]);
        float omega_local = den > 0.0f ? clamp_r(num / den, -om_abs, om_abs) : 0.0f;
        V2 g_eff = V2(0.0f, GRAVITY) + omega_local * omega_local * V2(sl[BS_XB], sl[BS_XB + 1]);
        V2 impulse = -rho_eff * K[BK_AREA] * g_eff * K[BK_DT];
        const float mass_l = K[BK_MASS];
        for (uint32_t s = lane; s < cnt; s += 32) {
          const uint32_t j = s < 32 ? q.j : BL.j[base + s];
          float frac = s < 32 ? q.frac : BL.w[base + s] / rho_local;
          V2 dv = -(impulse * frac) / mass_l;
          V_l[j] = (V2(V_l[j]) + dv).f2();
          if (s < 32) q.dv = dv;
          else if (want_mom) m.rec_M[BL.rec_off[b] + s] = (mass_l * dv).f2();
        }
        if (lane == 0) {
          float* slw = g_ball_slot[threadIdx.x >> 5];
          slw[BS_IMPULSE] = impulse.x;
          slw[BS_IMPULSE + 1] = impulse.y;
        }
      },
      // after the flag: the ball's impulse, the momentum records
      [&](uint32_t b, int lane, BuoyBall& q) {
        if (q.cnt == 0) return;
        if (want_mom && (uint32_t)lane < q.cnt) m.rec_M[BL.rec_off[b] + lane] = (m.f_mass * q.dv).f2();
        if (lane == 0) {
          const float* sl = g_ball_slot[threadIdx.x >> 5];
          m.imp[b] = (V2(m.imp[b]) + V2(sl[BS_IMPULSE], sl[BS_IMPULSE + 1])).f2();
        }
      });
}

// Step 6.6 (pbf.rs:2035-2122): the buoyancy sweep on the stale step-2 grid, in its own function
// like the drag sweep. beside: the helper blocks listed the items, records and claim order beside
// the drag sweep (WIDE_BESIDE_DRAG, still running); they are waited for first. Returns false when
// the item lists failed (the error is in *err).
static __device__ __noinline__ bool buoyancy_step(const MillDev& m, const StepUniform& U, StepOut& out,
                                                  uint32_t* err, FluidShared& S, float2* X, float2* V,
                                                  uint32_t* done, uint32_t* scratch, uint32_t scratch_words,
                                                  const uint32_t* drag_order, bool beside) {
  const uint32_t n = m.nf, nb = m.nb;
  if (beside) {
    wide_finish(m);
    const uint32_t n_items = wide_counter(m);
    if (tid() == 0) out.ctr.n_coupling_items += n_items;
    __syncthreads();
    if (*err) return false;
    stage_mark(out.stage, 27);
    const WideCtl* c = m.wide;
    const uint32_t nrec = c->beside_nrec;
    const uint32_t* order = c->beside_order_ok ? m.b_order : nullptr;
    stage_mark(out.stage, 28);
    buoyancy_sweep(m, U, out, err, X, V, done, order, BuoyLists{m.bi_n, m.bi_j, m.bi_w, m.bi_v, m.b_rec_off, m.b_rec_pred});
    if (tid() == 0 && U.want_momentum) {
      V2 mom(S.fscal[0], S.fscal[1]);
      for (uint32_t r = 0; r < nrec; ++r) mom += V2(m.rec_M[r]);
      S.fscal[0] = mom.x;
      S.fscal[1] = mom.y;
    }
    __syncthreads();
    stage_mark(out.stage, 29);
    return true;
  }
  if (nb > 0 && m.b_r > 0.0f) {
    uint32_t n_items = 0;
    wide_phase(m, WIDE_BUOYANCY_ITEMS, &S.hA, [&](uint32_t w0, uint32_t nw) {
      n_items += buoyancy_item_balls(m, S.hA, w0, nw, mill_items(m), m.item_n);
    });
    n_items = block_sum_u(n_items) + wide_counter(m);
    if (tid() == 0) out.ctr.n_coupling_items += n_items;
    __syncthreads();
    if (*err) return false;
    stage_mark(out.stage, 27);
    const uint32_t nrec = pack_ball_items(m.item_j, m.item_n, m.cap_items, nb, m.rec_off, m.rec_i, m.rec_b);
    // Claim order: a buoyancy item (a particle within h of the ball) is a drag item too (within
    // r + h), so every buoyancy predecessor is reached by a chain of drag predecessors and the drag
    // sweep's level order (when it ran) is topological here as well; it is checked all the same
    // (index order otherwise). Without a drag sweep, the buoyancy records' own levels.
    LevelScratch L;
    const bool by_level = U.sweep_order == 0 && level_scratch(nb, scratch, scratch_words, L);
    const bool reuse = by_level && drag_order != nullptr;
    ball_item_preds(m.rec_i, m.rec_b, nrec, n, nb, m.bk_start, m.bk_cur, m.bk_order, m.rec_pred,
                    by_level && !reuse ? &L : nullptr);
    const uint32_t* order = nullptr;
    if (reuse) order = order_respects(L.pos, m.rec_b, m.rec_pred, nrec) ? drag_order : nullptr;
    else if (by_level) order = ball_level_order(nb, m.rec_off, m.rec_pred, L);
    stage_mark(out.stage, 28);
    buoyancy_sweep(m, U, out, err, X, V, done, order,
                   BuoyLists{m.item_n, m.item_j, m.item_w, m.item_v, m.rec_off, m.rec_pred});
    if (tid() == 0 && U.want_momentum) {
      V2 mom(S.fscal[0], S.fscal[1]);
      for (uint32_t r = 0; r < nrec; ++r) mom += V2(m.rec_M[r]);
      S.fscal[0] = mom.x;
      S.fscal[1] = mom.y;
    }
    __syncthreads();
    stage_mark(out.stage, 29);
  }
  return true;
}

// Density recompute at the final positions X over the step-2 neighbour lists (pbf.rs:2132-2144).
static __device__ void density_recompute(const MillDev& m, const float2* X) {
  const uint32_t n = m.nf;
  const float h = m.f_h, mass = m.f_mass;
  const float self_rho = mass * poly6(0.0f, h);
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 xi(X[i]);
    float rho = self_rho;
    for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) rho += mass * poly6((xi - V2(X[m.nbrs[k]])).len2(), h);
    m.density[i] = rho;
  }
  __syncthreads();
}

// The viscosity's Morris weights and unit directions per edge (morris_weights, pbf.rs:312-345,
// called at pbf.rs:2154) from mu_eff and the recomputed densities at positions X.
static __device__ void morris_weights(const MillDev& m, const float2* X) {
  const uint32_t n = m.nf;
  const float h = m.f_h, mass = m.f_mass;
  const float eta2 = VISC_ETA * h * h;
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 xi(X[i]);
    float rho_i = fmax_r(m.density[i], 1e-6f);
    float mu_i = m.mu_eff[i];
    for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) {
      uint32_t j = m.nbrs[k];
      float rho_j = fmax_r(m.density[j], 1e-6f);
      V2 delta = xi - V2(X[j]);
      float r = delta.len();
      V2 grad = spiky_grad(delta, r, h);
      float numerator = (mass * (mu_i + m.mu_eff[j]) / (rho_i * rho_j)) * fabsf(delta.dot(grad));
      m.visc_w[k] = numerator / (delta.len2() + eta2);
      m.visc_dir[k] = (r > 1e-9f ? delta / r : V2(1.0f, 0.0f)).f2();
    }
  }
  __syncthreads();
}

// The boundary groups' per-particle factors (fluid_factor, pbf.rs:2172-2178, in f_tmp) and their
// fresh h-grid on X (pbf.rs:2163, header in hB).
static __device__ void group_factors_and_grid(const MillDev& m, const float2* X, GridHdr& hB, uint32_t* err) {
  const uint32_t n = m.nf;
  const float rho0 = m.f_rho0, mass = m.f_mass;
  grid_build(X, n, m.f_h, m.gB, hB, err);
  for (uint32_t j = tid(); j < n; j += nthr())
    m.f_tmp[j] = BALL_BC_GAIN * (mass * 2.0f * m.mu_eff[j] / (fmax_r(m.density[j], 1e-6f) * rho0));
  __syncthreads();
}

// The boundary groups in ball order from the per-ball lists I and the offsets g_off (scanned):
// fluid index, ball, coefficient, lever and squared lever per group (pbf.rs:2159-2232).
static __device__ void compact_groups(const MillDev& m, const ItemLists& I) {
  for (uint32_t b = tid() >> 5; b < m.nb; b += nthr() >> 5) {
    const uint32_t base = b * m.cap_items, o = m.g_off[b], cnt = m.g_off[b + 1] - o;
    for (uint32_t s = tid() & 31u; s < cnt; s += 32) {
      m.g_fluid[o + s] = I.j[base + s];
      m.g_ball[o + s] = b;
      m.g_c[o + s] = I.w[base + s];
      m.g_lc[o + s] = I.v[base + s];
      m.g_l2[o + s] = I.w2[base + s];
    }
  }
}

// Step 7 (pbf.rs:2146-2300): implicit viscosity on the velocities V at positions X (Morris weights,
// ball boundary groups, squeeze links, the fluid-only or joint fluid + ball CG and the ball
// impulses from it), in its own function so that it is register-allocated apart from the rest
// of the fluid step. visc_iters receives the CG iterations. Returns false when a capacity ran out
// or a grid failed (the error is in *err).
static __device__ __noinline__ bool viscosity_step(const MillDev& m, const StepUniform& U, StepOut& out,
                                                  uint32_t* err, FluidShared& S, float2* X, float2* V, float mu,
                                                  uint32_t& visc_iters, bool beside) {
  const uint32_t n = m.nf, nb = m.nb;
  const float h = m.f_h, mass = m.f_mass, dt = U.dt;
  const bool fp64 = U.cg_fp64 != 0;
  if (mu > 0.0f) {
    const bool bingham = U.slurry.rheology == MG_RHEOLOGY_BINGHAM && U.slurry.yield_stress_pa > 0.0f;
    const float tau_y = U.slurry.yield_stress_pa;
    // (beside: the helper blocks computed mu_eff, the Morris weights and the boundary groups'
    // lists beside the drag sweep)
    for (uint32_t i = tid(); !beside && i < n; i += nthr()) {
      float mu_i = mu;
      if (bingham) {
        // pbf.rs:821-868 shear rate then Papanastasiou viscosity
        V2 xi(X[i]), vi(V[i]);
        float gxx = 0.0f, gxy = 0.0f, gyx = 0.0f, gyy = 0.0f;
        for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) {
          uint32_t j = m.nbrs[k];
          V2 delta = xi - V2(X[j]);
          float r = delta.len();
          V2 grad = spiky_grad(delta, r, h);
          float coeff = mass / fmax_r(m.density[j], 1e-6f);
          V2 dv = V2(V[j]) - vi;
          gxx += coeff * dv.x * grad.x;
          gxy += coeff * dv.x * grad.y;
          gyx += coeff * dv.y * grad.x;
          gyy += coeff * dv.y * grad.y;
        }
        float dxy = 0.5f * (gxy + gyx);
        float g = sqrtf(2.0f * (gxx * gxx + gyy * gyy + 2.0f * dxy * dxy));
        float gamma0 = tau_y / (100.0f * mu);
        g = finite_f(g) ? g : 0.0f;
        float extra = g < 1e-4f * gamma0 ? tau_y / gamma0 : tau_y * (1.0f - expf_r(-g / gamma0)) / g;
        mu_i = mu + extra;
      }
      m.mu_eff[i] = mu_i;
    }
    __syncthreads();
    if (!beside) morris_weights(m, X);
    stage_mark(out.stage, 8);
    // boundary groups (pbf.rs:2159-2232) on a fresh h-grid, one ball per thread, merged per fluid
    if (tid() == 0) { S.n_groups = 0; S.n_links = 0; S.links_in_range = 0; }
    __syncthreads();
    if (nb > 0 && m.b_r > 0.0f) {
      const ItemLists I = beside ? ItemLists{m.gi_j, m.gi_v, m.gi_w, m.gi_w2} : mill_items(m);
      if (!beside) {
        group_factors_and_grid(m, X, S.hB, err);
        wide_phase(m, WIDE_GROUPS, &S.hB, [&](uint32_t w0, uint32_t nw) { group_balls(m, U, S.hB, w0, nw, I, w0); });
      }
      // (beside: helper block 1 compacted and sorted the groups unless something failed)
      const bool groups_sorted = beside && m.wide->beside_groups_ok != 0u;
      if (!groups_sorted && tid() == 0) m.g_off[nb] = 0;
      __syncthreads();
      if (*err) return false;
      if (groups_sorted) {
        if (tid() == 0) S.n_groups = m.wide->beside_ngroups;
      } else {
        uint32_t ng = block_exclusive_scan(m.g_off, nb + 1);
        if (ng > m.cap_groups) { if (tid() == 0) atomicOr(err, ERR_GROUPS); __syncthreads(); return false; }
        compact_groups(m, I);
        if (tid() == 0) S.n_groups = ng;
      }
      __syncthreads();
    }
    stage_mark(out.stage, 9);
    // ball_v0 (pbf.rs:2237-2239) and squeeze links (pbf.rs:544-625)
    for (uint32_t b = tid(); b < nb; b += nthr()) {
      m.ball_v0[b] = (V2(m.bv[b]) + V2(m.imp[b]) / m.b_m).f2();
      m.ball_w0[b] = m.bom[b] + m.ang[b] / m.b_I;
    }
    __syncthreads();
    if (nb > 0 && m.b_r > 0.0f) {
      const float r = m.b_r;
      const double dxd = (double)(0.5f * h);
      const float reach = (float)(8.0 * dxd);
      uint32_t tot_in = 0;
      // ball i's links go to its slots [i K, i K + K) of the record scratch, then one compaction
      // copies them to the link list in ball order. beside: the helper blocks listed the
      // candidates beside the drag sweep (unless a ball had more than its slots hold), so only the
      // velocity test is left.
      const uint32_t K = min(nb + 1u, 512u);
      if (beside && m.wide->beside_link_over == 0u) {
        tot_in = block_sum_u(links_from_candidates(m, tid() >> 5, nthr() >> 5));
      } else {
        uint32_t in_range = 0;
        grid_build(m.bx, nb, 2.0f * r + reach, m.gBall, S.hBall, err);
        wide_phase(m, WIDE_LINKS, &S.hBall,
                   [&](uint32_t w0, uint32_t nw) { in_range += link_balls(m, U, S.hBall, w0, nw); });
        tot_in = block_sum_u(in_range) + wide_counter(m);
      }
      if (tid() == 0) m.l_off[nb] = 0;
      __syncthreads();
      const uint32_t nl = block_exclusive_scan(m.l_off, nb + 1);
      if (nl > m.cap_links) { if (tid() == 0) atomicOr(err, ERR_LINKS); __syncthreads(); return false; }
      if (tid() == 0) { S.n_links = nl; S.links_in_range = tot_in; }
      for (uint32_t i = tid() >> 5; i < nb; i += nthr() >> 5) {
        const uint32_t o = m.l_off[i], cnt = m.l_off[i + 1] - o, base = i * K;
        for (uint32_t q = tid() & 31u; q < cnt; q += 32) {
          m.l_ball[o + q] = i;
          m.l_other[o + q] = m.rec_i[base + q];
          m.l_n[o + q] = m.rec_J[base + q];
          m.l_c[o + q] = m.rec_L[base + q];
        }
      }
      __syncthreads();
    }
    if (tid() == 0) {
      out.ctr.n_groups = S.n_groups;
      out.ctr.n_links = S.n_links;
      out.ctr.links_in_range = S.links_in_range;
    }
    __syncthreads();
    stage_mark(out.stage, 10);
    if (S.n_groups == 0 && S.links_in_range == 0) {
      // ---- fluid-only CG (pbf.rs:423-480), solution in place in V
      float2 *r = m.cg_r, *p = m.cg_p, *ap = m.cg_ap;
      double bn2 = block_dot(V, V, n, fp64, S);
      double b_norm = fp64 ? sqrt(bn2) : (double)sqrtf((float)bn2);
      if (b_norm > 0.0 && isfinite(b_norm)) {
        const float target_f = VISC_CG_TOL * (float)b_norm;
        const double target_d = (double)VISC_CG_TOL * b_norm;
        auto apply = [&](const float2* in, float2* o) {
          for (uint32_t i = tid(); i < n; i += nthr()) o[i] = (V2(in[i]) + dt * laplacian_row(m, in, i)).f2();
          __syncthreads();
        };
        apply(V, m.cg_ap);
        for (uint32_t i = tid(); i < n; i += nthr()) { r[i] = (V2(V[i]) - V2(ap[i])).f2(); p[i] = r[i]; }
        __syncthreads();
        double rs_old = block_dot(r, r, n, fp64, S);
        bool done = fp64 ? sqrt(rs_old) <= target_d : sqrtf((float)rs_old) <= target_f;
        if (!done) {
          visc_iters = VISC_CG_MAX;
          for (uint32_t it = 1; it <= VISC_CG_MAX; ++it) {
            apply(p, ap);
            double p_ap = block_dot(p, ap, n, fp64, S);
            if (p_ap <= 0.0 || !isfinite(p_ap)) { visc_iters = it; break; }
            float alpha = fp64 ? (float)(rs_old / p_ap) : (float)rs_old / (float)p_ap;
            for (uint32_t i = tid(); i < n; i += nthr()) {
              V[i] = (V2(V[i]) + alpha * V2(p[i])).f2();
              r[i] = (V2(r[i]) - alpha * V2(ap[i])).f2();
            }
            __syncthreads();
            double rs_new = block_dot(r, r, n, fp64, S);
            bool conv = fp64 ? sqrt(rs_new) <= target_d : sqrtf((float)rs_new) <= target_f;
            if (conv) { visc_iters = it; break; }
            float bt = fp64 ? (float)(rs_new / rs_old) : (float)rs_new / (float)rs_old;
            for (uint32_t i = tid(); i < n; i += nthr()) p[i] = (V2(r[i]) + bt * V2(p[i])).f2();
            __syncthreads();
            rs_old = rs_new;
          }
        }
      }
    } else {
      // ---- joint fluid + ball Jacobi-PCG (pbf.rs:641-791)
      const uint32_t len = n + 2 * nb;
      // per-fluid group lists and per-ball "other" link lists (stable, in group / link order)
      if (!(beside && m.wide->beside_groups_ok)) block_bucket_sort(m.g_fluid, S.n_groups, n, m.fg_start, m.bk_start, m.fg_list);
      for (uint32_t l = tid(); l < S.n_links; l += nthr()) m.rec_b[l] = m.l_other[l] == NONE ? nb : m.l_other[l];
      __syncthreads();
      // (bucket nb collects the links without a second ball; only the balls' lists are read)
      block_bucket_sort(m.rec_b, S.n_links, nb + 1, m.lo_start, m.bk_start, m.lo_list, nb);
      float2 *x = m.cg_x, *bvec = m.cg_b, *r = m.cg_r, *z = m.cg_z, *p = m.cg_p, *ap = m.cg_ap;
      float *diag = m.cg_diag, *inv = m.cg_inv;
      wide_phase(m, WIDE_CG_SETUP, nullptr, [&](uint32_t w0, uint32_t nw) {
        cg_setup_rows(m, dt, w0 * 32u + (tid() & 31u), nw * 32u);
      });
      for (uint32_t e = tid(); e < len; e += nthr()) inv[e] = 1.0f / fmax_r(diag[e], 1e-20f);
      __syncthreads();
      joint_apply(m, dt, x, ap);
      for (uint32_t e = tid(); e < len; e += nthr()) {
        V2 re = V2(bvec[e]) - V2(ap[e]);
        r[e] = re.f2();
        z[e] = (re * inv[e]).f2();
      }
      __syncthreads();
      double b_norm = block_res_norm(bvec, inv, len, fp64, S);
      double r_norm = block_res_norm(r, inv, len, fp64, S);
      stage_mark(out.stage, 23);
      double tol_b = fp64 ? (double)VISC_CG_TOL * b_norm : (double)(VISC_CG_TOL * (float)b_norm);
      if (b_norm > 0.0 && isfinite(b_norm) && r_norm > tol_b) {
        for (uint32_t e = tid(); e < len; e += nthr()) p[e] = z[e];
        __syncthreads();
        double rz_old = block_dot(r, z, len, fp64, S);
        for (uint32_t it = 1; it <= 4 * VISC_CG_MAX; ++it) {
          visc_iters = it;
          joint_apply(m, dt, p, ap);
          double p_ap = block_dot(p, ap, len, fp64, S);
          if (p_ap <= 0.0 || !isfinite(p_ap)) break;
          float alpha = fp64 ? (float)(rz_old / p_ap) : (float)rz_old / (float)p_ap;
          for (uint32_t e = tid(); e < len; e += nthr()) {
            x[e] = (V2(x[e]) + alpha * V2(p[e])).f2();
            r[e] = (V2(r[e]) - alpha * V2(ap[e])).f2();
          }
          __syncthreads();
          if (block_res_norm(r, inv, len, fp64, S) <= tol_b) break;
          for (uint32_t e = tid(); e < len; e += nthr()) z[e] = (V2(r[e]) * inv[e]).f2();
          __syncthreads();
          double rz_new = block_dot(r, z, len, fp64, S);
          float bt = fp64 ? (float)(rz_new / rz_old) : (float)rz_new / (float)rz_old;
          for (uint32_t e = tid(); e < len; e += nthr()) p[e] = (V2(z[e]) + bt * V2(p[e])).f2();
          __syncthreads();
          rz_old = rz_new;
        }
      }
      stage_mark(out.stage, 31);
      for (uint32_t i = tid(); i < n; i += nthr()) {
        V2 vn(x[i]);
        V[i] = vn.f2();
        V2 d = vn - V2(m.dv_tmp[i]);
        m.fguess[i] = (d.finite() ? d : V2()).f2();
      }
      __syncthreads();
      // ball impulses from the solved velocities (pbf.rs:2237-2298), one thread per ball
      for (uint32_t b = tid(); b < nb; b += nthr()) {
        V2 dv = V2(x[n + b]) - V2(m.ball_v0[b]);
        float dw = x[n + nb + b].x - m.ball_w0[b];
        if (dv.finite() && finite_f(dw)) {
          m.imp[b] = (V2(m.imp[b]) + m.b_m * dv).f2();
          m.ang[b] += m.b_I * dw;
        }
      }
      if (tid() == 0) m.guess_valid_dev[0] = 1u;
      if (U.want_momentum && tid() < 32) {
        // the fluid's momentum change loses b_m * dv per ball, in ball order (a - t == a + (-t))
        auto term = [&](uint32_t b, float& t, int c) {
          V2 dv = V2(x[n + b]) - V2(m.ball_v0[b]);
          float dw = x[n + nb + b].x - m.ball_w0[b];
          if (!(dv.finite() && finite_f(dw))) return false;
          V2 p = m.b_m * dv;
          t = -(c ? p.y : p.x);
          return true;
        };
        const float mx = warp_ordered_sum(S.fscal[0], nb, [&](uint32_t b, float& t) { return term(b, t, 0); });
        const float my = warp_ordered_sum(S.fscal[1], nb, [&](uint32_t b, float& t) { return term(b, t, 1); });
        if (tid() == 0) {
          S.fscal[0] = mx;
          S.fscal[1] = my;
        }
      }
      __syncthreads();
    }
  }
  return true;
}

// Steps 0-3 of the fluid sub-step (pbf.rs:1200-1334): sanitize, predict, the fluid grid and its
// neighbour lists, the density constraint iterations. They read and write only the fluid's arrays,
// so in a single-mill launch helper block 1 runs them for the next sub-step while the mill's block
// runs the DEM step (WIDE_FLUID_PREP). The grid header lands in S.hA and the edge count in
// S.n_edges; iters receives the density iterations and cycles[0..1] (thread 0) the clock cycles of
// steps 0-2 and of step 3. Returns early, with *err set, when the neighbour lists overflowed.
static __device__ void fluid_prep(const MillDev& m, uint32_t pbf_iterations, float dt, FluidShared& S,
                                  uint32_t* err, uint32_t& iters, unsigned long long* cycles) {
  const uint32_t n = m.nf;
  const float h = m.f_h, rho0 = m.f_rho0, mass = m.f_mass;
  float2* X = m.fx;
  float2* V = m.fv;
  const long long t0 = clock64();
  // ---- step 0: sanitize (pbf.rs:1200-1205)
  for (uint32_t i = tid(); i < n; i += nthr())
    if (!V2(X[i]).finite() || !V2(V[i]).finite()) { X[i] = make_float2(0.0f, 0.0f); V[i] = make_float2(0.0f, 0.0f); }
  __syncthreads();
  // ---- step 1: predict (pbf.rs:1225-1235)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 x(X[i]), v(V[i]);
    m.x0[i] = X[i];
    v.y += GRAVITY * dt;
    x += v * dt;
    X[i] = x.f2();
    V[i] = v.f2();
  }
  __syncthreads();
  // ---- step 2: grid + neighbour lists (pbf.rs:1238-1239)
  grid_build(X, n, h, m.gA, S.hA, err);
  build_neighbor_lists(X, n, h, S.hA, m.gA, m.nbr_off, m.nbrs, m.cap_edges, err, &S.n_edges);
  if (tid() == 0) cycles[0] = (unsigned long long)(clock64() - t0);
  // (block-uniform: on a helper block the mill's block may set *err at any time)
  if (__syncthreads_or(*err != 0u)) return;
  const long long t1 = clock64();
  // ---- step 3: density constraint (pbf.rs:1257-1334)
  const uint32_t base_it = pbf_iterations > 1 ? pbf_iterations : 1u;
  const float m_rho = mass / rho0;
  const float self_rho = mass * poly6(0.0f, h);
  uint32_t iter_count = 0;
  for (;;) {
    float max_c = 0.0f;
    for (uint32_t i = tid(); i < n; i += nthr()) {
      V2 xi(X[i]);
      float rho = self_rho;
      V2 grad_self;
      float sum_grad_sq = 0.0f;
      for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) {
        V2 delta = xi - V2(X[m.nbrs[k]]);
        float r2 = delta.len2();
        rho += mass * poly6(r2, h);
        float r = delta.len();
        V2 grad = spiky_grad(delta, r, h) * m_rho;
        grad_self += grad;
        sum_grad_sq += grad.len2();
      }
      m.density[i] = rho;
      float c_i = fmax_r(rho / rho0 - 1.0f, 0.0f);
      max_c = fmax_r(max_c, c_i);
      sum_grad_sq += grad_self.len2();
      m.lambda[i] = -c_i / (sum_grad_sq + EPSILON_RELAX);
    }
    max_c = block_max_f(max_c);
    for (uint32_t i = tid(); i < n; i += nthr()) {
      V2 xi(X[i]);
      float li = m.lambda[i];
      V2 sum;
      for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) {
        uint32_t j = m.nbrs[k];
        V2 delta = xi - V2(X[j]);
        float r = delta.len();
        sum += (li + m.lambda[j]) * spiky_grad(delta, r, h);
      }
      m.dp[i] = (sum * m_rho).f2();
    }
    __syncthreads();
    for (uint32_t i = tid(); i < n; i += nthr()) X[i] = (V2(X[i]) + V2(m.dp[i])).f2();
    __syncthreads();
    iter_count += 1;
    bool converged = max_c <= COMPRESSION_TOL;
    if ((iter_count >= base_it && converged) || iter_count >= base_it + ADAPTIVE_MAX_EXTRA) break;
  }
  if (tid() == 0) {
    iters = iter_count;
    cycles[1] = (unsigned long long)(clock64() - t1);
  }
}

// The fluid step's tail after the viscosity solve: the mean shear rate on the solved velocities
// (pbf.rs:800-849), then the speed clamp (pbf.rs:979-996, 2321), with the kinetic-energy terms of
// both (ke_mark: the fluid's kinetic energy before the solve). It reads and writes only the
// fluid's arrays and the three stats it sets in fs, and nothing later in the sub-step reads them,
// so in a single-mill launch helper block 1 runs it (ahead of the next sub-step's steps 0-3) while
// the mill's block runs the DEM step. Returns the clock cycles it took (thread 0).
static __device__ unsigned long long fluid_tail(const MillDev& m, float v_max, double ke_mark, MgFluidStepStats& fs,
                                                FluidShared& S) {
  const long long t0 = clock64();
  const uint32_t n = m.nf;
  const float h = m.f_h, mass = m.f_mass;
  const float2* X = m.fx;
  float2* V = m.fv;
  // ---- mean shear rate (pbf.rs:800-849) on the final velocities
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 xi(X[i]), vi(V[i]);
    float gxx = 0.0f, gxy = 0.0f, gyx = 0.0f, gyy = 0.0f;
    for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) {
      uint32_t j = m.nbrs[k];
      V2 delta = xi - V2(X[j]);
      float r = delta.len();
      V2 grad = spiky_grad(delta, r, h);
      float coeff = mass / fmax_r(m.density[j], 1e-6f);
      V2 dv = V2(V[j]) - vi;
      gxx += coeff * dv.x * grad.x;
      gxy += coeff * dv.x * grad.y;
      gyx += coeff * dv.y * grad.x;
      gyy += coeff * dv.y * grad.y;
    }
    float dxy = 0.5f * (gxy + gyx);
    m.f_tmp[i] = sqrtf(2.0f * (gxx * gxx + gyy * gyy + 2.0f * dxy * dxy));
  }
  __syncthreads();
  {
    const float s = block_seq_sum_f32<true>(0.0f, n, [&](uint32_t i) { return m.f_tmp[i]; });
    uint32_t c = 0;
    for (uint32_t i = tid(); i < n; i += nthr()) c += finite_f(m.f_tmp[i]) ? 1u : 0u;
    c = block_sum_u(c);
    if (tid() == 0) fs.mean_shear_rate_per_s = c == 0 ? 0.0f : s / (float)c;
  }
  __syncthreads();
  const double ke_after_visc = kinetic_energy_seq(V, n, mass, S);
  // ---- step 7.5: speed clamp (pbf.rs:979-996, 2321)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 v(V[i]);
    float speed = v.len();
    if (!finite_f(speed)) v = V2();
    else if (speed > v_max) v *= v_max / speed;
    V[i] = v.f2();
  }
  __syncthreads();
  const double ke_after_clamp = kinetic_energy_seq(V, n, mass, S);
  if (tid() == 0) {
    fs.ke_delta_viscosity_j = (float)(ke_after_visc - ke_mark);
    fs.ke_delta_clamp_j = (float)(ke_after_clamp - ke_after_visc);
  }
  __syncthreads();
  return (unsigned long long)(clock64() - t0);
}

// Helper blocks, WIDE_BESIDE_DRAG: the work that reads only the sub-step's final positions (after
// step 4) and nothing the drag sweep writes, done while the mill's block runs the drag sweep. The
// tasks the mill's block asked for (BESIDE_*) are split by helper block:
//   * block 1 (BESIDE_VISC): the density recompute (pbf.rs:2132-2144), mu_eff = mu and the Morris
//     weights (pbf.rs:2146-2154), the boundary groups' per-particle factors and h-grid, whose
//     header it publishes for the other helpers right after building it; then (BESIDE_BUOY), once
//     every other helper has listed its buoyancy items, the buoyancy records, their predecessor
//     balls and a claim order by dependency level (as buoyancy_step does without a drag order);
//   * blocks 2..: their shares of the buoyancy item lists (pbf.rs:2042-2060) into bi_*, counted
//     in the phase's counter, then, once the grid is published, of the boundary groups
//     (pbf.rs:2159-2232) into gi_* and g_off.
// The waits between helpers are bounded like the mill's (ERR_WIDE; the waiting block then skips
// the work that needed the other).
static __device__ uint32_t beside_drag(const MillDev& m, const StepUniform& U, const GridHdr& hA, FluidShared& S,
                                       unsigned char* dsm) {
  __shared__ uint32_t ok;
  WideCtl* c = m.wide;
  const uint32_t tasks = c->beside_tasks;
  const uint32_t n = m.nf, nb = m.nb;
  const float2* X = m.fx;
  const long long lim = m.wide_wait_cycles > 0 ? m.wide_wait_cycles : WIDE_TIMEOUT_CYCLES;
  if (blockIdx.x == 1) {
    if (tasks & BESIDE_VISC) {
      density_recompute(m, X);
      const float mu = c->beside_mu;
      for (uint32_t i = tid(); i < n; i += nthr()) m.mu_eff[i] = mu;
      __syncthreads();
      group_factors_and_grid(m, X, S.hB, m.err);
      if (nb > 0 && m.b_r > 0.0f)  // the squeeze links' ball grid (pbf.rs:544-560)
        grid_build(m.bx, nb, 2.0f * m.b_r + (float)(8.0 * (double)(0.5f * m.f_h)), m.gBall, S.hBall, m.err);
      if (tid() == 0) {
        c->beside_hdr = S.hB;
        c->beside_link_hdr = S.hBall;
        __threadfence();
        *reinterpret_cast<volatile uint32_t*>(&c->beside_grid_seq) = 1u;
      }
      morris_weights(m, X);
    }
    if (tasks & BESIDE_BUOY) {
      if (tid() == 0) {
        ok = wide_wait(&c->beside_buoy_blocks, m.helpers - 1u, lim) ? 1u : 0u;
        if (!ok) atomicOr(m.err, ERR_WIDE);
        __threadfence();
      }
      __syncthreads();
      if (ok) {
        const uint32_t nrec = pack_ball_items(m.bi_j, m.bi_n, m.cap_items, nb, m.b_rec_off, m.b_rec_i, m.b_rec_b);
        LevelScratch L;
        const bool by_level = U.sweep_order == 0 &&
                              level_scratch(nb, reinterpret_cast<uint32_t*>(dsm), m.smem_bytes / 4u, L);
        ball_item_preds(m.b_rec_i, m.b_rec_b, nrec, n, nb, m.hb_start, m.hb_cur, m.hb_order, m.b_rec_pred,
                        by_level ? &L : nullptr);
        if (by_level) {
          const uint32_t* order = ball_level_order(nb, m.b_rec_off, m.b_rec_pred, L);
          for (uint32_t b = tid(); b < nb; b += nthr()) m.b_order[b] = order[b];
        }
        if (tid() == 0) {
          c->beside_nrec = nrec;
          c->beside_order_ok = by_level ? 1u : 0u;
        }
        __syncthreads();
      }
    }
    if (tasks & BESIDE_VISC) {
      // the boundary groups in ball order (their lists compacted from gi_*) and their per-fluid
      // lists (a stable bucket sort by fluid particle), once every helper has listed its share
      if (tid() == 0) {
        ok = wide_wait(&c->beside_group_blocks, m.helpers - 1u, lim) ? 1u : 0u;
        if (!ok) atomicOr(m.err, ERR_WIDE);
        __threadfence();
        if (*reinterpret_cast<volatile uint32_t*>(m.err) != 0u) ok = 0u;
        m.g_off[nb] = 0;
      }
      __syncthreads();
      if (ok) {
        const uint32_t ng = block_exclusive_scan(m.g_off, nb + 1);
        if (ng > m.cap_groups) {
          if (tid() == 0) atomicOr(m.err, ERR_GROUPS);
        } else {
          compact_groups(m, ItemLists{m.gi_j, m.gi_v, m.gi_w, m.gi_w2});
          __syncthreads();
          block_bucket_sort(m.g_fluid, ng, n, m.fg_start, m.hb_cur, m.fg_list);
          if (tid() == 0) {
            c->beside_ngroups = ng;
            c->beside_groups_ok = 1u;
          }
        }
        __syncthreads();
      }
    }
    return 0u;
  }
  const uint32_t nwarps = nthr() >> 5, warp = tid() >> 5;
  const uint32_t w0 = (blockIdx.x - 2u) * nwarps + warp, nw = (m.helpers - 1u) * nwarps;
  uint32_t items = 0;
  if (tasks & BESIDE_BUOY) {
    items = buoyancy_item_balls(m, hA, w0, nw, ItemLists{m.bi_j, m.bi_v, m.bi_w, nullptr}, m.bi_n);
    __syncthreads();
    if (tid() == 0) {
      __threadfence();
      atomicAdd(&c->beside_buoy_blocks, 1u);
    }
  }
  if (tasks & BESIDE_VISC) {
    if (tid() == 0) {
      ok = wide_wait(&c->beside_grid_seq, 1u, lim) ? 1u : 0u;
      if (!ok) atomicOr(m.err, ERR_WIDE);
      __threadfence();
      S.hB = c->beside_hdr;
      S.hBall = c->beside_link_hdr;
    }
    __syncthreads();
    if (ok) group_balls(m, U, S.hB, w0, nw, ItemLists{m.gi_j, m.gi_v, m.gi_w, m.gi_w2}, blockIdx.x * nwarps + warp);
    __syncthreads();
    if (tid() == 0) {
      __threadfence();
      atomicAdd(&c->beside_group_blocks, 1u);
    }
    if (ok && nb > 0 && m.b_r > 0.0f) link_candidate_balls(m, U, S.hBall, w0, nw, &c->beside_link_over);
  }
  return items;
}

// Helper blocks, WIDE_DRAG_LISTS: the drag sweep's inputs, which read only the final positions,
// listed while the mill's block runs steps 5-6 (velocity reconstruction and wall no-slip, which
// write only velocities). Helper block 1 builds the drag grid (cell r + h, pbf.rs:1794-1796) and
// publishes its header; helper blocks 2.. then list their shares of the item lists
// (drag_item_balls) and the per-ball pre-sums (drag_pre_balls) and count themselves done; helper
// block 1 then packs the records, their predecessor balls and, by dependency level, the claim order
// into d_order. The phase's counter receives the item count. Waits between helpers are bounded
// (ERR_WIDE).
static __device__ uint32_t drag_lists(const MillDev& m, const StepUniform& U, FluidShared& S, unsigned char* dsm) {
  __shared__ uint32_t ok;
  WideCtl* c = m.wide;
  const uint32_t n = m.nf, nb = m.nb;
  const long long lim = m.wide_wait_cycles > 0 ? m.wide_wait_cycles : WIDE_TIMEOUT_CYCLES;
  if (blockIdx.x == 1) {
    const float h_c = m.b_r + m.f_h;
    grid_build(m.fx, n, fmax_r(h_c, 1e-6f), m.gB, S.hB, m.err);
    if (tid() == 0) {
      c->drag_hdr = S.hB;
      __threadfence();
      *reinterpret_cast<volatile uint32_t*>(&c->drag_grid_seq) = 1u;
      ok = wide_wait(&c->drag_blocks, m.helpers - 1u, lim) ? 1u : 0u;
      if (!ok) atomicOr(m.err, ERR_WIDE);
      __threadfence();
    }
    __syncthreads();
    if (ok) {
      const uint32_t nrec = pack_ball_items(m.item_j, m.item_n, m.cap_items, nb, m.rec_off, m.rec_i, m.rec_b);
      LevelScratch L;
      const bool by_level =
          U.sweep_order == 0 && level_scratch(nb, reinterpret_cast<uint32_t*>(dsm), m.smem_bytes / 4u, L);
      ball_item_preds(m.rec_i, m.rec_b, nrec, n, nb, m.bk_start, m.bk_cur, m.bk_order, m.rec_pred,
                      by_level ? &L : nullptr);
      if (by_level) {
        const uint32_t* order = ball_level_order(nb, m.rec_off, m.rec_pred, L);
        for (uint32_t b = tid(); b < nb; b += nthr()) m.d_order[b] = order[b];
      }
      if (tid() == 0) c->drag_order_ok = by_level ? 1u : 0u;
      __syncthreads();
    }
    return 0u;
  }
  if (tid() == 0) {
    ok = wide_wait(&c->drag_grid_seq, 1u, lim) ? 1u : 0u;
    if (!ok) atomicOr(m.err, ERR_WIDE);
    __threadfence();
    S.hB = c->drag_hdr;
  }
  __syncthreads();
  uint32_t items = 0;
  if (ok) {
    const uint32_t nwarps = nthr() >> 5;
    const uint32_t w0 = (blockIdx.x - 2u) * nwarps + (tid() >> 5), nw = (m.helpers - 1u) * nwarps;
    items = drag_item_balls(m, S.hB, w0, nw);
    __syncwarp();
    drag_pre_balls(m, w0, nw);  // the same balls, from the lists this warp just wrote
  }
  __syncthreads();
  if (tid() == 0) {
    __threadfence();
    atomicAdd(&c->drag_blocks, 1u);
  }
  return items;
}

// Step 4's wall accumulations in particle order (pbf.rs:1635-1653), by warp 0: each lane keeps one
// angle bin of the normal impulse; every lane carries the three f64 impulse sums (identical
// chains), left in S.dscal[0..2]. Its own function, so that the unrolled shuffle loops are
// register-allocated apart from the fluid step around them (inlined there they spilled).
static __device__ __noinline__ void wall_sums_step4(const MillDev& m, uint32_t n, StepOut& out, FluidShared& S) {
  if (tid() < 32) {
    const int lane = tid();
    float bin_acc = 0.0f;
    double ix = 0.0, iy = 0.0, ia = 0.0;
    // the three f64 sums by the order-free exact path when it applies (same bits), else below
    const bool exact = warp_exact_sum_f64(0.0, n, [&](uint32_t i, double& t) {
                         if (m.wall_bin[i] < 0) return false; t = (double)m.dv_tmp[i].x; return true; }, ix) &&
                       warp_exact_sum_f64(0.0, n, [&](uint32_t i, double& t) {
                         if (m.wall_bin[i] < 0) return false; t = (double)m.dv_tmp[i].y; return true; }, iy) &&
                       warp_exact_sum_f64(0.0, n, [&](uint32_t i, double& t) {
                         if (m.wall_bin[i] < 0) return false; t = (double)m.f_tmp[i]; return true; }, ia);
    if (!exact) ix = iy = ia = 0.0;
    for (uint32_t c = 0; c < n; c += 32) {
      int32_t bin = -1;
      float val = 0.0f, px = 0.0f, py = 0.0f, pa = 0.0f;
      if (c + lane < n) {
        bin = m.wall_bin[c + lane];
        if (bin >= 0) { val = m.wall_val[c + lane]; px = m.dv_tmp[c + lane].x; py = m.dv_tmp[c + lane].y; pa = m.f_tmp[c + lane]; }
      }
      const uint32_t mask = __ballot_sync(FULL, bin >= 0);
      if (mask == 0u) continue;  // no particle of the chunk touched the wall
      if (exact) {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
          const int bt = __shfl_sync(FULL, bin, t);
          const float vt = __shfl_sync(FULL, val, t);
          if (((mask >> t) & 1u) && bt == lane) bin_acc += vt;
        }
        continue;
      }
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const int bt = __shfl_sync(FULL, bin, t);
        const float vt = __shfl_sync(FULL, val, t), xt = __shfl_sync(FULL, px, t), yt = __shfl_sync(FULL, py, t);
        const float at = __shfl_sync(FULL, pa, t);
        if ((mask >> t) & 1u) {
          ix += (double)xt;
          iy += (double)yt;
          ia += (double)at;
          if (bt == lane) bin_acc += vt;
        }
      }
    }
    out.fs.wall_normal_impulse_by_angle[lane] = bin_acc;
    if (lane == 0) { S.dscal[0] = ix; S.dscal[1] = iy; S.dscal[2] = ia; }
  }
}

// Step 6's accumulations in particle order (pbf.rs:1677-1700), continuing the step-4 impulse sums in
// S.dscal[0..2], and the wall work into out.fs.wall_work_j, by warp 0. Its own function, like
// wall_sums_step4.
static __device__ __noinline__ void wall_sums_step6(const MillDev& m, const StepUniform& U, const float2* X,
                                                    uint32_t n, float mass, StepOut& out, FluidShared& S) {
  if (tid() < 32) {
    const int lane = tid();
    float work = 0.0f;
    double ix = S.dscal[0], iy = S.dscal[1], ia = S.dscal[2];
    // the three f64 sums by the order-free exact path when it applies (same bits), else below
    double ex_ix, ex_iy, ex_ia;
    const bool exact =
        warp_exact_sum_f64(ix, n, [&](uint32_t i, double& t) {
          if (m.wall_bin[i] < 0) return false; t = (double)(mass * V2(m.dv_tmp[i]).x); return true; }, ex_ix) &&
        warp_exact_sum_f64(iy, n, [&](uint32_t i, double& t) {
          if (m.wall_bin[i] < 0) return false; t = (double)(mass * V2(m.dv_tmp[i]).y); return true; }, ex_iy) &&
        warp_exact_sum_f64(ia, n, [&](uint32_t i, double& t) {
          if (m.wall_bin[i] < 0) return false; t = (double)cross2(V2(X[i]), mass * V2(m.dv_tmp[i])); return true; }, ex_ia);
    for (uint32_t c = 0; c < n; c += 32) {
      bool touched = c + lane < n && m.wall_bin[c + lane] >= 0;
      float wk = 0.0f, jx = 0.0f, jy = 0.0f, ja = 0.0f;
      if (touched) {
        V2 x(X[c + lane]);
        V2 dv(m.dv_tmp[c + lane]);
        wk = mass * dv.dot(wall_velocity(U.drum_omega, x));
        jx = mass * dv.x;
        jy = mass * dv.y;
        ja = cross2(x, mass * dv);
      }
      const uint32_t mask = __ballot_sync(FULL, touched);
      if (mask == 0u) continue;
      if (exact) {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
          const float wt = __shfl_sync(FULL, wk, t);
          if ((mask >> t) & 1u) work += wt;
        }
        continue;
      }
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const float wt = __shfl_sync(FULL, wk, t), xt = __shfl_sync(FULL, jx, t), yt = __shfl_sync(FULL, jy, t);
        const float at = __shfl_sync(FULL, ja, t);
        if ((mask >> t) & 1u) {
          work += wt;
          ix += (double)xt;
          iy += (double)yt;
          ia += (double)at;
        }
      }
    }
    __syncwarp();
    if (exact) {
      ix = ex_ix;
      iy = ex_iy;
      ia = ex_ia;
    }
    if (lane == 0) { S.dscal[0] = ix; S.dscal[1] = iy; S.dscal[2] = ia; out.fs.wall_work_j = work; }
  }
}

// defer_tail: leave fluid_tail to helper block 1 (the caller publishes it). Returns whether the
// tail was left out; *ke_tail then receives its ke_mark argument.
static __device__ bool fluid_step(const MillDev& m, const StepUniform& U, StepOut& out, uint32_t* err, FluidShared& S,
                                  unsigned char* dsm, bool prepped, bool defer_tail, double* ke_tail) {
  if (prepped) wide_finish(m);   // helper block 1 ran steps 0-3 (published with WIDE_FLUID_PREP)
  uint32_t* done = m.ball_done;  // completion flags of the per-ball sweeps (moved to shared below)
  const uint32_t n = m.nf, nb = m.nb;
  const float dt = U.dt;
  for (uint32_t b = tid(); b < nb; b += nthr()) { m.imp[b] = make_float2(0.0f, 0.0f); m.ang[b] = 0.0f; }
  if (tid() == 0) { memset(&out.fs, 0, sizeof(out.fs)); out.clamp_hits = 0; out.fluid_momentum[0] = out.fluid_momentum[1] = 0.0f; }
  __syncthreads();
  if (n == 0 || dt <= 0.0f) return false;
  const float h = m.f_h, rho0 = m.f_rho0, mass = m.f_mass;
  float2* X = m.fx;
  float2* V = m.fv;
  if (prepped) {
    // steps 0-3 ran on helper block 1 during the previous sub-step's DEM step: take over the
    // fluid grid's header and the counts
    if (tid() == 0) {
      const WideCtl* c = m.wide;
      if (c->prep_err) atomicOr(err, c->prep_err);
      S.hA = c->prep_hdr;
      S.n_edges = c->prep_edges;
      out.ctr.n_fluid_edges = c->prep_edges;
      out.ctr.density_iters = c->prep_iters;
      out.stage[0] += c->prep_cycles[0];
      out.stage[1] += c->prep_cycles[1];
    }
    __syncthreads();
    if (*err) return false;
  } else {
    uint32_t iters = 0;
    unsigned long long cyc[2] = {0, 0};
    stage_mark(out.stage, 0);
    fluid_prep(m, U.pbf_iterations, dt, S, err, iters, cyc);
    if (tid() == 0) {
      out.ctr.n_fluid_edges = S.n_edges;
      out.ctr.density_iters = iters;
      out.stage[0] += cyc[0];
      out.stage[1] += cyc[1];
      g_stage_last = clock64();
    }
    __syncthreads();
    if (*err) return false;
  }
  // ball grid for the overlap push (pbf.rs:1214-1222); it reads only the balls, so it comes after
  // steps 0-3 here
  const float contact_radius = m.b_r + OVERLAP_PUSH_MARGIN * h;
  if (nb > 0) grid_build(m.bx, nb, fmax_r(fmax_r(2.0f * m.b_r, contact_radius), 1e-6f), m.gBall, S.hBall, err);
  stage_mark(out.stage, 0);
  // ---- step 3.5: ball overlap push (pbf.rs:1361-1444); two passes (count, fill), then the
  // per-ball reaction sums replayed in the reference's (fluid index, near order) order.
  for (uint32_t i = tid(); i < n; i += nthr()) m.push_ex[i] = make_float2(0.0f, 0.0f);
  if (nb > 0) {
    const float reduced_mass = m.b_m > 0.0f ? (mass * m.b_m) / (mass + m.b_m) : mass;
    for (int pass = 0; pass < 2; ++pass) {
      for (uint32_t i = tid(); i < n; i += nthr()) {
        V2 xi(X[i]);
        V2 vi(V[i]);
        V2 ex;
        uint32_t c = 0, o = pass ? m.rec_cnt[i] : 0;
        V2 xq = xi;
        for_each_near(S.hBall, m.gBall, xq, [&](uint32_t b) {
          V2 delta = xi - V2(m.bx[b]);
          float dist = delta.len();
          if (isnan_f(dist) || dist >= contact_radius) return;
          V2 n_hat = dist > 1e-9f ? delta / dist : V2(1.0f, 0.0f);
          float push_mag = fmin_r(contact_radius - dist, 0.5f * m.b_r);
          xi += push_mag * n_hat;
          V2 lever = n_hat * m.b_r;
          V2 v_surface = V2(m.bv[b]) + m.bom[b] * V2(-lever.y, lever.x);
          float arrest = fmax_r(-(vi - v_surface).dot(n_hat), 0.0f);
          float full = mass * push_mag / dt;
          float imag = fmin_r(full, reduced_mass * arrest);
          ex += ((full - imag) / mass) * n_hat;
          if (pass) {
            V2 reaction = -imag * n_hat;
            if (o < m.cap_recs) {
              m.rec_i[o] = i;
              m.rec_b[o] = b;
              m.rec_J[o] = reaction.f2();
              m.rec_L[o] = cross2(lever, reaction);
              m.rec_M[o] = (imag * n_hat).f2();
            }
            ++o;
          }
          ++c;
        });
        if (!pass) {
          m.rec_cnt[i] = c;
        } else {
          X[i] = xi.f2();
          m.push_ex[i] = ex.f2();
        }
      }
      __syncthreads();
      if (!pass) {
        if (tid() == 0) m.rec_cnt[n] = 0;
        __syncthreads();
        S.n_recs = 0;
        uint32_t tot = block_exclusive_scan(m.rec_cnt, n + 1);
        if (tot > m.cap_recs) { if (tid() == 0) atomicOr(err, ERR_RECORDS); __syncthreads(); return false; }
        if (tid() == 0) S.n_recs = tot;
        __syncthreads();
      }
    }
    // per-ball reaction sums in record order (fluid index ascending, near order): a stable
    // bucket sort of the records by ball, then one thread per ball
    block_bucket_sort(m.rec_b, S.n_recs, nb, m.bk_start, m.bk_cur, m.bk_order);
    for (uint32_t b = tid(); b < nb; b += nthr()) {
      V2 J;
      float L = 0.0f;
      for (uint32_t q = m.bk_start[b]; q < m.bk_start[b + 1]; ++q) {
        uint32_t r = m.bk_order[q];
        J += V2(m.rec_J[r]);
        L += m.rec_L[r];
      }
      m.imp[b] = J.f2();
      m.ang[b] = L;
    }
    if (tid() == 0) {
      V2 mom;
      if (U.want_momentum)
        for (uint32_t q = 0; q < S.n_recs; ++q) mom += V2(m.rec_M[q]);
      S.fscal[0] = mom.x;
      S.fscal[1] = mom.y;
    }
  } else if (tid() == 0) {
    S.fscal[0] = S.fscal[1] = 0.0f;
  }
  __syncthreads();
  stage_mark(out.stage, 2);
  // ---- step 3.6a: cohesion (pbf.rs:1464-1491)
  const float cohesion_accel = (fmax_r(U.slurry.surface_tension_n_m, 0.0f) / 0.072f) * 2.0f * fabsf(GRAVITY);
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 pull;
    if (cohesion_accel > 0.0f) {
      V2 xi(X[i]);
      for (uint32_t k = m.nbr_off[i]; k < m.nbr_off[i + 1]; ++k) {
        V2 delta = xi - V2(X[m.nbrs[k]]);
        float r = delta.len();
        if (r <= 1e-9f) continue;
        float w = mass * cohesion_kernel(r, h) / rho0;
        pull -= w * (delta / r);
      }
      m.coh_dv[i] = (cohesion_accel * pull * dt).f2();
    } else {
      m.coh_dv[i] = make_float2(0.0f, 0.0f);
    }
    m.adh_dv[i] = make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  stage_mark(out.stage, 3);
  // ---- step 3.6b: adhesion (pbf.rs:1515-1631) on the stale step-2 grid
  const float wett = clamp_r(U.slurry.wettability, 0.0f, 1.0f);
  const uint32_t count_pb = U.boundary_count;
  if (wett > 0.0f && nb > 0 && m.b_r > 0.0f && count_pb > 0) {
    const float h_adh = fmin_r(h, 2.0f * m.b_r);
    if (h_adh > 0.0f) {
      wide_phase(m, WIDE_ADHESION, &S.hA, [&](uint32_t w0, uint32_t nw) { adhesion_balls(m, U, S.hA, w0, nw); });
      __syncthreads();
      if (*err) return false;
      // per-fluid sums of the balls' contributions in ball order (stable bucket sort by fluid)
      uint32_t nrec = pack_ball_items(m.item_j, m.item_n, m.cap_items, nb, m.rec_off, m.rec_i, m.rec_b);
      for (uint32_t b = tid() >> 5; b < nb; b += nthr() >> 5) {
        const uint32_t o = m.rec_off[b], base = b * m.cap_items, cnt = m.item_n[b];
        for (uint32_t s = tid() & 31u; s < cnt; s += 32) m.rec_J[o + s] = m.item_v[base + s];
      }
      __syncthreads();
      block_bucket_sort(m.rec_i, nrec, n, m.bk_start, m.bk_cur, m.bk_order);
      for (uint32_t j = tid(); j < n; j += nthr()) {
        V2 acc;
        for (uint32_t q = m.bk_start[j]; q < m.bk_start[j + 1]; ++q) acc += V2(m.rec_J[m.bk_order[q]]);
        if (m.bk_start[j + 1] > m.bk_start[j]) m.adh_dv[j] = acc.f2();
      }
      if (tid() == 0 && U.want_momentum) {
        V2 mom(S.fscal[0], S.fscal[1]);
        for (uint32_t r = 0; r < nrec; ++r) mom += mass * V2(m.rec_J[r]);
        S.fscal[0] = mom.x;
        S.fscal[1] = mom.y;
      }
      __syncthreads();
    }
  }
  stage_mark(out.stage, 4);
  // ---- step 4: wall projection (pbf.rs:1635-1653)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 x(X[i]), pl;
    // the normal only for particles outside the wall; interior particles skip the lifters
    const float d = x.finite() && drum_sdf_clear(U, rotate(x, U.to_local_next), 0.0f)
                        ? 0.0f : drum_sdf_world_dist(U, x, U.to_local_next, pl);
    if (d < 0.0f) {
      const V2 normal = drum_sdf_world_normal(U, x, pl, U.to_world_next);
      x += -d * normal;
      X[i] = x.f2();
      V2 push = mass * (-d * normal) / dt;
      m.dv_tmp[i] = push.f2();
      m.f_tmp[i] = cross2(x, push);
      float angle = atan2f_r(x.y, x.x);
      uint32_t bin = f2u_sat(((angle + PI_F) / TAU_F) * 32.0f);
      m.wall_bin[i] = (int32_t)(bin < 31u ? bin : 31u);
      m.wall_val[i] = mass * -d / dt;
    } else {
      m.wall_bin[i] = -1;
    }
  }
  __syncthreads();
  // The positions are final from here on: with two or more helper blocks and a drag sweep to run,
  // the helpers list the drag sweep's items, records and claim order (drag_lists) while this
  // block runs steps 5-6.
  bool drag_listed = false;
  {
    const float mu_d = fmax_r(U.slurry.viscosity_pa_s, 0.0f);
    if (m.helpers >= 2 && m.d_order != nullptr && nb > 0 && m.b_r > 0.0f && m.b_rtrue > 0.0f && mu_d > 1e-6f &&
        clamp_r(U.slurry.ball_no_slip, 0.0f, 1.0f) > 0.0f) {
      wide_publish(m, WIDE_DRAG_LISTS, nullptr, nullptr, nullptr, [&](WideCtl* c) {
        c->drag_grid_seq = 0u;
        c->drag_blocks = 0u;
        c->drag_order_ok = 0u;
      });
      drag_listed = true;
    }
  }
  // accumulations in particle order by warp 0 (wall_sums_step4)
  wall_sums_step4(m, n, out, S);
  __syncthreads();
  // ---- step 5: velocity reconstruction (pbf.rs:1656-1674)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 v = (V2(X[i]) - V2(m.x0[i])) / dt;
    v -= V2(m.push_ex[i]);
    v += V2(m.coh_dv[i]);
    v += V2(m.adh_dv[i]);
    V[i] = v.f2();
  }
  __syncthreads();
  // ---- step 6: wall no-slip (pbf.rs:1677-1700)
  const float beta = clamp_r(U.slurry.wall_no_slip, 0.0f, 1.0f);
  double ke_before_noslip = kinetic_energy_seq(V, n, mass, S);
  if (beta > 0.0f) {
    for (uint32_t i = tid(); i < n; i += nthr()) {
      if (m.wall_bin[i] < 0) continue;
      V2 x(X[i]);
      V2 v_wall = wall_velocity(U.drum_omega, x);
      V2 v_old(V[i]);
      V2 v = (1.0f - beta) * v_old + beta * v_wall;
      V[i] = v.f2();
      m.dv_tmp[i] = (v - v_old).f2();
    }
    __syncthreads();
    // accumulations in particle order, continuing the step-4 sums (warp 0: wall_sums_step6)
    wall_sums_step6(m, U, X, n, mass, out, S);
    __syncthreads();
  }
  double ke_mark = kinetic_energy_seq(V, n, mass, S);
  const double ke_delta_noslip = ke_mark - ke_before_noslip;
  stage_mark(out.stage, 5);
  // The drag and buoyancy sweeps (steps 6.5 / 6.6) run on copies of X and V in the dynamic shared
  // region when they fit, with the per-ball completion flags after them; V is written back after
  // step 6.6. X does not change in between.
  float2* Vg = V;
  float2* Xg = X;
  uint32_t* sweep_scratch = nullptr;  // the rest of the region: the sweeps' claim orders
  uint32_t sweep_words = 0;
  if (16u * n + 4u * nb + 64u <= m.smem_bytes) {
    float2* sX = reinterpret_cast<float2*>(dsm);
    float2* sV = sX + n;
    for (uint32_t i = tid(); i < n; i += nthr()) { sX[i] = Xg[i]; sV[i] = Vg[i]; }
    done = reinterpret_cast<uint32_t*>(sV + n);
    sweep_scratch = done + nb;
    sweep_words = (m.smem_bytes - (16u * n + 4u * nb)) / 4u;
    X = sX;
    V = sV;
    __syncthreads();
  } else {
    done = m.ball_done;
  }
  // ---- step 6.5: ball drag, Gauss-Seidel over balls (pbf.rs:1777-2013)
  const float mu = fmax_r(U.slurry.viscosity_pa_s, 0.0f);
  const uint32_t* drag_order = nullptr;  // the drag sweep's claim order, when it ran by level
  uint32_t beside = 0;  // BESIDE_* parts the helper blocks do beside the drag sweep
  if (!drag_step(m, U, out, err, S, X, V, done, sweep_scratch, sweep_words, &drag_order, &beside, drag_listed))
    return false;
  stage_mark(out.stage, 19);
  double ke_after_drag = kinetic_energy_seq(V, n, mass, S);
  const double ke_delta_drag = ke_after_drag - ke_mark;
  ke_mark = ke_after_drag;
  // ---- step 6.6: buoyancy, Gauss-Seidel over balls on the stale step-2 grid (pbf.rs:2035-2122)
  if (!buoyancy_step(m, U, out, err, S, X, V, done, sweep_scratch, sweep_words, drag_order,
                     (beside & BESIDE_BUOY) != 0u))
    return false;
  double ke_after_buoy = kinetic_energy_seq(V, n, mass, S);
  const double ke_delta_buoy = ke_after_buoy - ke_mark;
  ke_mark = ke_after_buoy;
  if (V != Vg) {
    for (uint32_t i = tid(); i < n; i += nthr()) Vg[i] = V[i];
    V = Vg;
    X = Xg;
    __syncthreads();
  }
  stage_mark(out.stage, 6);
  // ---- density recompute at final x over the step-2 lists (the helper blocks did it beside the
  // drag sweep with BESIDE_VISC)
  if (!(beside & BESIDE_VISC)) density_recompute(m, X);
  stage_mark(out.stage, 7);
  // ---- step 7: implicit viscosity (pbf.rs:2146-2300)
  uint32_t visc_iters = 0;
  if (!viscosity_step(m, U, out, err, S, X, V, mu, visc_iters, (beside & BESIDE_VISC) != 0u)) return false;
  stage_mark(out.stage, 11);
  // ---- mean shear rate and step 7.5, the speed clamp (fluid_tail); they touch nothing that
  // step 8 or the DEM step reads
  if (defer_tail) {
    *ke_tail = ke_mark;
  } else {
    const unsigned long long cyc = fluid_tail(m, fluid_vmax(U), ke_mark, out.fs, S);
    if (tid() == 0) {
      out.stage[12] += cyc;
      g_stage_last = clock64();
    }
  }
  // ---- step 8: impulse clamp (pbf.rs:2330-2345)
  uint32_t hits = 0;
  if (nb > 0) {
    const float clamp = 60.0f * m.b_m * 9.81f * dt;
    const float angular_clamp = clamp * m.b_r;
    for (uint32_t b = tid(); b < nb; b += nthr()) {
      V2 J(m.imp[b]);
      float mag = J.len();
      if (mag > clamp && mag > 1e-9f) { J *= clamp / mag; hits += 1; }
      m.imp[b] = J.f2();
      m.ang[b] = clamp_r(m.ang[b], -angular_clamp, angular_clamp);
    }
  }
  hits = block_sum_u(hits);
  if (tid() == 0) {
    out.ctr.cg_iters = visc_iters;
    out.fs.viscosity_iterations = visc_iters;
    out.fs.coupling_clamp_hits = hits;
    out.clamp_hits = hits;
    out.fs.wall_impulse[0] = (float)S.dscal[0];
    out.fs.wall_impulse[1] = (float)S.dscal[1];
    out.fs.wall_angular_impulse = (float)S.dscal[2];
    out.fs.ke_delta_noslip_j = (float)ke_delta_noslip;
    out.fs.ke_delta_drag_j = (float)ke_delta_drag;
    out.fs.ke_delta_buoyancy_j = (float)ke_delta_buoy;
    out.fluid_momentum[0] = S.fscal[0];
    out.fluid_momentum[1] = S.fscal[1];
  }
  __syncthreads();
  stage_mark(out.stage, 13);
  return defer_tail;
}

}  // namespace mg
