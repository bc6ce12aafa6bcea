// metrics::compute (metrics.rs:195-273) on the device: one block reads a mill's current state
// and fills an MgMetrics. Sums keep the reference's order (block_seq_sum_f32), maxima and minima
// are exact selections, and the angle lists are sorted stably, so every field is the same bits
// as the sequential computation.
#pragma once

#include "mill_fluid.cuh"

namespace mg {

constexpr float MET_WALL_MARGIN_BALL_RADII = 2.5f;            // metrics.rs:37
constexpr uint32_t MET_MIN_WALL_BALLS = 6;                    // metrics.rs:41
constexpr float MET_CENTRIFUGE_GAP_RAD = PI_F * 0.3f;         // metrics.rs:45
constexpr float MET_POOL_WALL_MARGIN_H = 1.5f;                // metrics.rs:48
constexpr float MET_POOL_DEPTH_BAND_RAD = 5.0f * PI_F / 180.0f;  // metrics.rs:51
constexpr int MET_MIXING_GRID = 16;                           // metrics.rs:62

__device__ __forceinline__ float met_rem_euclid(float x, float m) {
  const float r = fmodf(x, m);
  return r < 0.0f ? r + fabsf(m) : r;
}
// p.y.atan2(p.x).rem_euclid(TAU)
__device__ __forceinline__ float met_world_angle(V2 p) { return met_rem_euclid(atan2f_r(p.y, p.x), TAU_F); }

__device__ inline float block_min_f(float v) {
  __shared__ float sh[32];
  __shared__ float res;
  for (int o = 16; o > 0; o >>= 1) v = fmin_r(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = tid() >> 5, l = tid() & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    const int nw = (nthr() + 31) >> 5;
    float x = l < nw ? sh[l] : INFINITY;
    for (int o = 16; o > 0; o >>= 1) x = fmin_r(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (l == 0) res = x;
  }
  __syncthreads();
  const float r = res;
  __syncthreads();
  return r;
}

// Writes val(i) for the i < n with pred(i), in index order, to dst; returns their count.
template <class Pred, class Val, class T>
__device__ uint32_t met_compact(uint32_t n, uint32_t* flags, T* dst, Pred pred, Val val) {
  for (uint32_t i = tid(); i < n; i += nthr()) flags[i] = pred(i) ? 1u : 0u;
  if (tid() == 0) flags[n] = 0;
  __syncthreads();
  const uint32_t k = block_exclusive_scan(flags, n + 1);
  for (uint32_t i = tid(); i < n; i += nthr())
    if (flags[i + 1] != flags[i]) dst[flags[i]] = val(i);
  __syncthreads();
  return k;
}

// Stable ascending sort of src[0..k) into dst (sort_by(partial_cmp): equal values, -0.0 and 0.0
// included, keep their order), by rank counting.
static __device__ void met_rank_sort(const float* src, float* dst, uint32_t k) {
  for (uint32_t i = tid(); i < k; i += nthr()) {
    const float a = src[i];
    uint32_t r = 0;
    for (uint32_t j = 0; j < k; ++j) {
      const float b = src[j];
      r += (b < a || (b == a && j < i)) ? 1u : 0u;
    }
    dst[r] = a;
  }
  __syncthreads();
}

// metrics.rs:292-307 over sorted angles a[0..n), n >= 2 (one thread).
static __device__ void met_largest_gap(const float* a, uint32_t n, float* start, float* end, float* gap) {
  float max_gap = a[0] + TAU_F - a[n - 1];
  uint32_t gap_k = n - 1;
  for (uint32_t i = 0; i + 1 < n; ++i) {
    const float g = a[i + 1] - a[i];
    if (g > max_gap) {
      max_gap = g;
      gap_k = i;
    }
  }
  *end = a[gap_k];
  *start = a[(gap_k + 1) % n];
  *gap = max_gap;
}

// One block of up to 1024 threads; mills[0] is the mill, uni its uniform block with to_local_next /
// to_world_next set to the current drum angle's rotations.
__global__ void __launch_bounds__(1024) metrics_kernel(const MillDev* __restrict__ mills,
                                                        const StepUniform* __restrict__ uni, MgMetrics* out) {
  __shared__ MillDev m;
  __shared__ GridHdr hdr;
  __shared__ MgMetrics o;
  if (tid() == 0) {
    m = mills[0];
    memset(&o, 0, sizeof(o));
  }
  __syncthreads();
  const StepUniform& U = *uni;
  const uint32_t nb = m.nb, nf = m.nf;
  const float r = m.b_r, h = m.f_h;
  auto wall_d = [&](V2 p) {
    V2 pl;
    return drum_sdf_world_dist(U, p, U.to_local_next, pl);
  };
  float* A = m.cg_diag;  // angle lists (n + 2 nb >= both populations)
  float* B = m.cg_inv;   // sorted
  uint32_t* flags = m.act_flag;    // ball flags (nb + 1)
  uint32_t* fflags = m.rec_cnt;    // fluid flags (nf + 1)
  if (nb > 0) {
    // charge_toe_shoulder (metrics.rs:327-360)
    const float margin = MET_WALL_MARGIN_BALL_RADII * r;
    const uint32_t k = met_compact(nb, flags, A, [&](uint32_t i) { return wall_d(V2(m.bx[i])) < margin; },
                                   [&](uint32_t i) { return met_world_angle(V2(m.bx[i])); });
    if (k >= MET_MIN_WALL_BALLS) {
      met_rank_sort(A, B, k);
      if (tid() == 0) {
        float cs, ce, gap;
        met_largest_gap(B, k, &cs, &ce, &gap);
        if (!(gap <= MET_CENTRIFUGE_GAP_RAD)) {
          o.valid |= MG_METRIC_TOE_SHOULDER;
          o.toe_angle_rad = U.drum_omega >= 0.0f ? cs : ce;
          o.shoulder_angle_rad = U.drum_omega >= 0.0f ? ce : cs;
        }
      }
    }
    // charge_centroid (metrics.rs:362-369)
    const float sx = block_seq_sum_f32(0.0f, nb, [&](uint32_t i) { return m.bx[i].x; });
    const float sy = block_seq_sum_f32(0.0f, nb, [&](uint32_t i) { return m.bx[i].y; });
    if (tid() == 0) {
      const V2 c = V2(sx, sy) / (float)nb;
      o.valid |= MG_METRIC_CENTROID;
      o.charge_centroid_m[0] = c.x;
      o.charge_centroid_m[1] = c.y;
    }
    // total_kinetic_energy_j (metrics.rs:581-590)
    const float b_m = m.b_m, b_I = m.b_I;
    const float ke = block_seq_sum_f32(0.0f, nb, [&](uint32_t i) {
      const float w = m.bom[i];
      return 0.5f * b_m * V2(m.bv[i]).len2() + 0.5f * b_I * w * w;
    });
    if (tid() == 0) o.total_kinetic_energy_j = ke;
    // max_ball_wall_overlap_fraction (metrics.rs:621-634)
    if (r > 0.0f) {
      float mw = 0.0f;
      for (uint32_t i = tid(); i < nb; i += nthr()) mw = fmax_r(mw, fmax_r(r - wall_d(V2(m.bx[i])), 0.0f) / r);
      mw = block_max_f(mw);
      if (tid() == 0) o.max_ball_wall_overlap_fraction = mw;
    }
    // max_ball_overlap_fraction (metrics.rs:599-612): every pair closer than 2r lies in the same or
    // an adjacent cell of a 2r * 1.05 grid, and the max over them does not depend on the order
    if (nb >= 2 && r > 0.0f) {
      grid_build(m.bx, nb, fmax_r(2.0f * r * 1.05f, 1e-6f), m.gBall, hdr, m.err);
      float mo = 0.0f;
      for (uint32_t i = tid(); i < nb; i += nthr()) {
        const V2 xi(m.bx[i]);
        for_each_near(hdr, m.gBall, xi, [&](uint32_t j) {
          if (j == i) return;
          const float dist = (xi - V2(m.bx[j])).len();
          mo = fmax_r(mo, fmax_r(2.0f * r - dist, 0.0f) / r);
        });
      }
      mo = block_max_f(mo);
      if (tid() == 0) o.max_ball_overlap_fraction = mo;
    }
  }
  if (nf > 0) {
    const float margin = MET_POOL_WALL_MARGIN_H * h;
    // slurry_pool_angular_extent (metrics.rs:377-400)
    const uint32_t k = met_compact(nf, fflags, A, [&](uint32_t i) { return wall_d(V2(m.fx[i])) < margin; },
                                   [&](uint32_t i) { return met_world_angle(V2(m.fx[i])); });
    if (k == 1 && tid() == 0) {
      o.valid |= MG_METRIC_POOL_EXTENT;
      o.pool_angle_min_rad = o.pool_angle_max_rad = A[0];
    } else if (k >= 2) {
      met_rank_sort(A, B, k);
      if (tid() == 0) {
        float cs, ce, gap;
        met_largest_gap(B, k, &cs, &ce, &gap);
        o.valid |= MG_METRIC_POOL_EXTENT;
        o.pool_angle_min_rad = cs;
        o.pool_angle_max_rad = ce;
      }
    }
    __syncthreads();
    // fluid_free_surface_line (metrics.rs:414-461) over the particles away from the wall
    uint32_t* idx = m.rec_i;
    const uint32_t kp = met_compact(nf, fflags, idx, [&](uint32_t i) { return wall_d(V2(m.fx[i])) >= margin; },
                                    [&](uint32_t i) { return i; });
    if (kp >= 3) {
      const float n = (float)kp;
      const float sx = block_seq_sum_f32(0.0f, kp, [&](uint32_t q) { return m.fx[idx[q]].x; });
      const float sy = block_seq_sum_f32(0.0f, kp, [&](uint32_t q) { return m.fx[idx[q]].y; });
      const V2 c = V2(sx, sy) / n;
      float cxx = block_seq_sum_f32(0.0f, kp, [&](uint32_t q) { const float e = m.fx[idx[q]].x - c.x; return e * e; });
      float cyy = block_seq_sum_f32(0.0f, kp, [&](uint32_t q) { const float e = m.fx[idx[q]].y - c.y; return e * e; });
      float cxy = block_seq_sum_f32(0.0f, kp, [&](uint32_t q) {
        const V2 e = V2(m.fx[idx[q]]) - c;
        return e.x * e.y;
      });
      if (tid() == 0) {
        cxx /= n;
        cyy /= n;
        cxy /= n;
        const float angle = 0.5f * atan2f_r(2.0f * cxy, cxx - cyy);
        const V2 normal(-sinf_r(angle), cosf_r(angle));
        o.valid |= MG_METRIC_FREE_SURFACE;
        o.free_surface_angle_rad = angle;
        o.free_surface_offset_m = c.dot(normal);
      }
    }
    // slurry_pool_depth_at_bottom (metrics.rs:463-477)
    const float down = 3.0f * (0.5f * PI_F);
    float md = INFINITY;
    uint32_t in_band = 0;
    for (uint32_t i = tid(); i < nf; i += nthr()) {
      const V2 p(m.fx[i]);
      const float d = met_rem_euclid(met_world_angle(p) - down, TAU_F);
      if (fmin_r(d, TAU_F - d) <= MET_POOL_DEPTH_BAND_RAD) {
        md = fmin_r(md, p.len());
        in_band += 1;
      }
    }
    md = block_min_f(md);
    in_band = block_sum_u(in_band);
    if (tid() == 0 && in_band > 0) {
      o.valid |= MG_METRIC_POOL_DEPTH;
      o.pool_depth_m = U.drum_radius - md;
    }
    // mixing_index (metrics.rs:506-576): per-cell dye sums in particle order
    const float R = U.drum_radius;
    if (R > 0.0f) {
      constexpr int G = MET_MIXING_GRID;
      const float cell = 2.0f * R / (float)G;
      for (uint32_t i = tid(); i < nf; i += nthr()) {
        const V2 p(m.fx[i]);
        const int32_t gi = min(max(f2i_sat(floorf((p.x + R) / cell)), 0), G - 1);
        const int32_t gj = min(max(f2i_sat(floorf((p.y + R) / cell)), 0), G - 1);
        idx[i] = (uint32_t)(gj * G + gi);
      }
      __syncthreads();
      __shared__ uint32_t cstart[G * G + 1], ccur[G * G];
      __shared__ float cell_sum[G * G];
      block_bucket_sort(idx, nf, G * G, cstart, ccur, m.bk_order);
      for (uint32_t c = tid(); c < (uint32_t)(G * G); c += nthr()) {
        float s = 0.0f;
        for (uint32_t q = cstart[c]; q < cstart[c + 1]; ++q) s += m.fdye[m.bk_order[q]];
        cell_sum[c] = s;
      }
      const float total = block_seq_sum_f32(0.0f, nf, [&](uint32_t i) { return m.fdye[i]; });
      if (tid() == 0) {
        const float p_mean = total / (float)nf;
        uint32_t cells = 0, ws = 0;
        for (int c = 0; c < G * G; ++c) {
          const uint32_t cnt = cstart[c + 1] - cstart[c];
          if (cnt) { cells += 1; ws += cnt; }
        }
        if (cells >= 2) {
          const float wsum = (float)ws;
          float ov = 0.0f, wa = 0.0f;
          for (int c = 0; c < G * G; ++c) {
            const uint32_t cnt = cstart[c + 1] - cstart[c];
            if (!cnt) continue;
            const float dm = cell_sum[c] / (float)cnt - p_mean;
            ov += (float)cnt * (dm * dm);
          }
          for (int c = 0; c < G * G; ++c) {
            const uint32_t cnt = cstart[c + 1] - cstart[c];
            if (cnt) wa += (float)cnt * (float)cnt;
          }
          const float observed = ov / wsum;
          const float s0 = p_mean * (1.0f - p_mean);
          const float sr = s0 / fmax_r(wa / wsum, 1.0f);
          if (!(s0 < 1e-9f)) {
            const float denom = s0 - sr;
            o.valid |= MG_METRIC_MIXING;
            o.mixing_index = fabsf(denom) < 1e-9f ? 1.0f : clamp_r((s0 - observed) / denom, 0.0f, 1.0f);
          }
        }
      }
      __syncthreads();
    }
    // fluid density errors (metrics.rs:649-711) on FluidParticles::densities (pbf.rs:1124-1141):
    // each particle's density adds its neighbours in candidate-pair order, which is the order of
    // its neighbour list
    // (the densities themselves are left in m.f_tmp for mg_fluid_densities)
    const float rest = m.f_rho0;
    grid_build(m.fx, nf, h, m.gA, hdr, m.err);
    __shared__ uint32_t n_edges;
    build_neighbor_lists(m.fx, nf, h, hdr, m.gA, m.nbr_off, m.nbrs, m.cap_edges, m.err, &n_edges);
    const float mass = m.f_mass;
    const float self_c = mass * poly6(0.0f, h);
    float* rho = m.f_tmp;
    for (uint32_t i = tid(); i < nf; i += nthr()) {
      const V2 xi(m.fx[i]);
      float d = self_c;
      for (uint32_t q = m.nbr_off[i]; q < m.nbr_off[i + 1]; ++q) d += mass * poly6((xi - V2(m.fx[m.nbrs[q]])).len2(), h);
      rho[i] = d;
    }
    __syncthreads();
    if (rest > 0.0f) {
      float mx = 0.0f, cmx = 0.0f;
      for (uint32_t i = tid(); i < nf; i += nthr()) {
        mx = fmax_r(mx, fabsf(rho[i] - rest) / rest);
        cmx = fmax_r(cmx, fmax_r(rho[i] / rest - 1.0f, 0.0f));
      }
      mx = block_max_f(mx);
      cmx = block_max_f(cmx);
      const float sm = block_seq_sum_f32(0.0f, nf, [&](uint32_t i) { return fabsf(rho[i] - rest) / rest; });
      const float csm = block_seq_sum_f32(0.0f, nf, [&](uint32_t i) { return fmax_r(rho[i] / rest - 1.0f, 0.0f); });
      if (tid() == 0) {
        o.valid |= MG_METRIC_DENSITY;
        o.max_fluid_density_error_fraction = mx;
        o.mean_fluid_density_error_fraction = sm / (float)nf;
        o.max_fluid_compression_error_fraction = cmx;
        o.mean_fluid_compression_error_fraction = csm / (float)nf;
      }
    }
  }
  __syncthreads();
  if (tid() == 0) {
    o.drum_omega_rad_s = U.drum_omega;
    o.fluid_particle_count = nf;
    *out = o;
  }
}

}  // namespace mg
