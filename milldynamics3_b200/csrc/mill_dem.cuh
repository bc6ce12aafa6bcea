// The ball half of the sub-step (DemState::step_recorded, dem.rs:530-1066) for one mill, executed
// by one thread block. Per-ball stages run in parallel; the broad phase materialises the candidate
// pairs in the grid's visiting order; the Gauss-Seidel projection, friction and restitution sweeps
// are replayed exactly (mill_replay.cuh): the projection by dependency levels, the contact sweeps
// in 32-item chunks. Ball state lives in shared memory during the sweeps when it fits.
#pragma once

#include "mill_geom.cuh"
#include "mill_grid.cuh"
#include "mill_replay.cuh"

namespace mg {

constexpr float RESTITUTION_VELOCITY_THRESHOLD = 0.02f;
constexpr float MAX_RECOVERY_FRACTION = 0.2f;
constexpr float CCD_SKIN_FRACTION = 1e-2f;
// projection runs over a subset of the pairs before the last one runs all of them
constexpr uint32_t PROJECTION_ROUNDS = 4;

struct DemShared {
  GridHdr hg;
  uint32_t npairs, nact, nrec_imp, collisions;
  uint32_t hist[MG_IMPACT_BINS];
  float fscal[4];
  double dscal[4];
};

// dem.rs:1071-1080 (the wrap loops are bounded; a difference beyond 1024 turns is flagged)
__device__ __forceinline__ float angle_diff(float a, float b, uint32_t* err) {
  float d = a - b;
  int guard = 0;
  while (d > PI_F && guard < 1024) { d -= 2.0f * PI_F; ++guard; }
  while (d < -PI_F && guard < 2048) { d += 2.0f * PI_F; ++guard; }
  if (guard >= 1024) atomicOr(err, ERR_BUDGET);
  return d;
}

// dem.rs:127-138
__device__ __forceinline__ float effective_friction(float mu_k, float mu_s, float v_t, float vs) {
  if (mu_s <= mu_k) return mu_k;
  float ratio = v_t / vs;
  float weight = expf_r(-(ratio * ratio));
  return mu_k + (mu_s - mu_k) * weight;
}

// dem.rs:99-109 (-1 for None)
__device__ __forceinline__ int impact_energy_bin(float e) {
  if (!finite_f(e) || e <= 0.0f) return -1;
  float ec = clamp_r(e, 1e-6f, 1.0f);
  float log_min = log10f_r(1e-6f);
  float log_max = log10f_r(1.0f);
  float t = (log10f_r(ec) - log_min) / (log_max - log_min);
  uint32_t idx = f2u_sat(t * 12.0f);
  return (int)(idx < 11u ? idx : 11u);
}

// dem.rs:253-261 f32 mechanical energy, summed in ball order (three adds per ball); called by
// warp 0, result in every lane
static __device__ __noinline__ float mech_energy_seq(const MillDev& m, const float2* X, const float2* V, const float* OM) {
  const uint32_t lane = threadIdx.x & 31u;
  float e = 0.0f;
  for (uint32_t c = 0; c < m.nb; c += 32) {
    float a = 0.0f, b = 0.0f, g = 0.0f;
    uint32_t i = c + lane;
    if (i < m.nb) {
      a = 0.5f * m.b_m * V2(V[i]).len2();
      b = 0.5f * m.b_I * OM[i] * OM[i];
      g = m.b_m * fabsf(GRAVITY) * X[i].y;
    }
    uint32_t lim = min(32u, m.nb - c);
#pragma unroll
    for (uint32_t t = 0; t < 32; ++t) {
      const float at = __shfl_sync(FULL, a, t), bt = __shfl_sync(FULL, b, t), gt = __shfl_sync(FULL, g, t);
      if (t < lim) {
        e += at;
        e += bt;
        e += gt;
      }
    }
  }
  return e;
}

// The predict step's coupling work summed in ball order in f64 (dem.rs:577-586), by warp 0 (result
// in every lane). Its own function, so that the unrolled shuffle loop does not spill.
static __device__ __noinline__ double coupling_work_seq(const MillDev& m) {
  return warp_ordered_sum(0.0, m.nb, [&](uint32_t i, double& t) { t = m.f_cw[i]; return true; });
}

// `iters` iterations of the projection (dem.rs:711-750): the pair items by dependency levels in
// warp 0 (level-ordered descriptors di/dj, multipliers dl), then every wall at once. With track,
// bm[i] keeps ball i's largest squared excursion from its start position m.bxs[i]. Its own
// function, so that the item bodies are register-allocated apart from the step around them.
static __device__ __noinline__ void project_iterations(const MillDev& m, const StepUniform& U, float2* X, float* dl,
                                                       float* bm, const uint32_t* di, const uint32_t* dj,
                                                       uint32_t nlev, uint32_t iters, uint32_t n, bool track, float r,
                                                       float w, float cap_depth) {
  // the larger of the recorded and the new squared excursion; a NaN excursion is kept (and
  // fails the check)
  auto excursion = [](float cur, V2 d) {
    const float e = d.len2();
    return !(e <= cur) ? e : cur;
  };
  float2* const Xp = X;
  float* const dlp = dl;
  const float2* const bxs = m.bxs;
  float* const bmv = bm;
  const uint32_t* const dip = di;
  const uint32_t* const djp = dj;
  for (uint32_t it = 0; it < iters; ++it) {
    run_levels(nlev, m.lev_start, [dip, djp](uint32_t q) { return make_uint2(dip[q], djp[q]); },
               [Xp, dlp, bxs, bmv, track, r, w, cap_depth, excursion](uint32_t q, uint2 d) {
      float2* const X = Xp;
      float* const dl = dlp;
      const uint32_t i = d.x, j = d.y;
      V2 xi(X[i]), xj(X[j]);
      const float dlq = dl[q];  // loaded beside the positions (only this item writes it)
      // start positions and excursions so far, loaded beside the positions
      V2 si, sj;
      float ei = 0.0f, ej = 0.0f;
      if (track) { si = V2(bxs[i]); sj = V2(bxs[j]); ei = bmv[i]; ej = bmv[j]; }
      V2 delta = xi - xj;
      float dist = delta.len();
      float c = dist - 2.0f * r;
      if (c >= 0.0f) return;
      V2 n_hat = dist > 1e-9f ? delta / dist : V2(1.0f, 0.0f);
      float w_sum = w + w;
      if (w_sum <= 0.0f) return;
      float c_eff = fmax_r(c, cap_depth);
      float d_lambda = -c_eff / w_sum;
      const V2 xin = xi + w * d_lambda * n_hat, xjn = xj - w * d_lambda * n_hat;
      X[i] = xin.f2();
      X[j] = xjn.f2();
      dl[q] = dlq + d_lambda;
      if (track) {
        bmv[i] = excursion(ei, V2(xin.f2()) - si);
        bmv[j] = excursion(ej, V2(xjn.f2()) - sj);
      }
    });
    for (uint32_t i = tid(); i < n; i += nthr()) {
      V2 x(X[i]), pl;
      if (x.finite() && drum_sdf_clear(U, rotate(x, U.to_local_next), r)) continue;  // c >= 0 certainly
      float d = drum_sdf_world_dist(U, x, U.to_local_next, pl);
      float c = d - r;
      if (c >= 0.0f) continue;
      if (w <= 0.0f) continue;
      V2 n_hat = drum_sdf_world_normal(U, x, pl, U.to_world_next);
      float c_eff = fmax_r(c, cap_depth);
      float d_lambda = -c_eff / w;
      const V2 xn = x + w * d_lambda * n_hat;
      X[i] = xn.f2();
      m.lam_bw[i] += d_lambda;
      if (track) bm[i] = excursion(bm[i], V2(xn.f2()) - V2(m.bxs[i]));
    }
    __syncthreads();
  }
}

// Step 5 friction sweep (dem.rs:782-882) over the active contacts in sweep order: the pair contacts
// by dependency levels in warp 0 (contacts of one level share no ball), then the wall contacts
// (every wall contact comes after every pair contact and touches one ball) at once. Wall contacts
// leave their work terms in act_w1 / act_w2 (act_bin -2: none). Its own function, like
// project_iterations.
static __device__ __noinline__ void friction_sweep(const MillDev& m, const StepUniform& U, float2* X, float2* V,
                                                   float* TH, float* OM, uint32_t nlev_c, uint32_t na_p, uint32_t na,
                                                   float w, float w_rot, float r, float dt) {
  // the sweep's constants, read once (the per-item bodies keep them in registers)
  const float mu_bb = U.media.friction_ball_ball, mu_bb_s = U.media.friction_ball_ball_static;
  const float mu_bw = U.media.friction_ball_wall, mu_bw_s = U.media.friction_ball_wall_static;
  const float vscale = U.media.friction_velocity_scale_m_s;
  const float w_sum_pair = w + w + r * r * w_rot + r * r * w_rot;
  const float w_sum_wall = w + r * r * w_rot;
  float2* const X_l = X;
  float2* const V_l = V;
  float* const TH_l = TH;
  float* const OM_l = OM;
  // pair contacts by dependency levels in warp 0
  run_levels(nlev_c, m.lev_start,
             [&](uint32_t q) {
               const uint32_t k = m.lev_items[q];
               return make_uint3(m.act_i[k], m.act_j[k], __float_as_uint(m.act_l[k]));
             },
             [&](uint32_t, uint3 d) {
               const uint32_t i = d.x, j = d.y;
               const float lambda_n = __uint_as_float(d.z);
               V2 delta = V2(X_l[i]) - V2(X_l[j]);
               float dist = delta.len();
               V2 n_hat = dist > 1e-9f ? delta / dist : V2(1.0f, 0.0f);
               V2 t_hat(-n_hat.y, n_hat.x);
               float v_t = (V2(V_l[i]) - V2(V_l[j])).dot(t_hat) - r * OM_l[i] - r * OM_l[j];
               if (w_sum_pair <= 0.0f) return;
               float raw = -v_t * dt / w_sum_pair;
               float mu = effective_friction(mu_bb, mu_bb_s, v_t, vscale);
               float max_mag = mu * lambda_n;
               float dlt = clamp_r(raw, -max_mag, max_mag);
               X_l[i] = (V2(X_l[i]) + w * dlt * t_hat).f2();
               X_l[j] = (V2(X_l[j]) - w * dlt * t_hat).f2();
               TH_l[i] -= r * w_rot * dlt;
               TH_l[j] -= r * w_rot * dlt;
               V2 dv = w * dlt * t_hat / dt;
               float domega = -r * w_rot * dlt / dt;
               V_l[i] = (V2(V_l[i]) + dv).f2();
               V_l[j] = (V2(V_l[j]) - dv).f2();
               OM_l[i] += domega;
               OM_l[j] += domega;
             });
  // then the wall contacts, each on its own ball, all at once
  for (uint32_t k = na_p + tid(); k < na; k += nthr()) {
    const uint32_t i = m.act_i[k];
    const float lambda_n = m.act_l[k];
    m.act_bin[k] = -2;  // no work terms unless the contact completes below
    float dd;
    V2 n_hat;
    drum_sdf_world(U, V2(X_l[i]), U.to_local_next, U.to_world_next, dd, n_hat);
    V2 t_hat(-n_hat.y, n_hat.x);
    V2 v_wall = wall_velocity(U.drum_omega, V2(X_l[i]) - r * n_hat);
    float v_t = (V2(V_l[i]) - v_wall).dot(t_hat) - r * OM_l[i];
    if (w_sum_wall <= 0.0f) continue;
    float raw = -v_t * dt / w_sum_wall;
    float mu = effective_friction(mu_bw, mu_bw_s, v_t, vscale);
    float max_mag = mu * lambda_n;
    float dlt = clamp_r(raw, -max_mag, max_mag);
    X_l[i] = (V2(X_l[i]) + w * dlt * t_hat).f2();
    TH_l[i] -= r * w_rot * dlt;
    V_l[i] = (V2(V_l[i]) + w * dlt * t_hat / dt).f2();
    OM_l[i] += -r * w_rot * dlt / dt;
    m.act_w1[k] = (dlt / dt) * t_hat.dot(v_wall);
    m.act_w2[k] = (lambda_n / dt) * n_hat.dot(v_wall);
    m.act_bin[k] = 0;
  }
  __syncthreads();
}

// Step 6 restitution sweep (dem.rs:909-1019) over the active contacts, with the impact accounting
// (collision count and energy histogram in S, impact records flagged in act_flag / act_rec).
// Positions do not change in this sweep, so each pair contact's normal, approach speed, impact
// accounting and target normal speed are computed for all pair contacts at once (act_w1 / act_w2 /
// act_t); the pair chain then only reads and updates the two velocities. The wall contacts come
// after every pair contact, each on its own ball, all at once.
static __device__ __noinline__ void restitution_sweep(const MillDev& m, const StepUniform& U, DemShared& S, float2* X,
                                                      float2* V, uint32_t nlev_c, uint32_t na_p, uint32_t na, float w,
                                                      float r, float impact_threshold) {
  const float e_bb = U.media.restitution_ball_ball, e_bw = U.media.restitution_ball_wall;
  for (uint32_t k = tid(); k < na_p; k += nthr()) {
    const uint32_t i = m.act_i[k], j = m.act_j[k];
    m.act_flag[k] = 0;
    V2 delta = V2(X[i]) - V2(X[j]);
    float dist = delta.len();
    V2 n_hat = dist > 1e-9f ? delta / dist : V2(1.0f, 0.0f);
    float v_n_pre = (V2(m.bvpre[i]) - V2(m.bvpre[j])).dot(n_hat);
    bool fresh = v_n_pre < -RESTITUTION_VELOCITY_THRESHOLD;
    if (fresh) {
      atomicAdd(&S.collisions, 1u);
      int bin = impact_energy_bin(0.5f * (m.b_m * 0.5f) * v_n_pre * v_n_pre);
      if (bin >= 0) atomicAdd(&S.hist[bin], 1u);
    }
    float e = fresh ? e_bb : 0.0f;
    if (-v_n_pre > impact_threshold) {
      V2 t_hat(-n_hat.y, n_hat.x);
      float slip = (V2(m.bvpre[i]) - V2(m.bvpre[j])).dot(t_hat) - r * m.bompre[i] - r * m.bompre[j];
      m.act_rec[k] = MgImpactRecord{MG_IMPACT_BALL_BALL, i, j, -v_n_pre, fabsf(slip), e};
      m.act_flag[k] = 1;
    }
    m.act_w1[k] = n_hat.x;
    m.act_w2[k] = n_hat.y;
    m.act_t[k] = fmax_r(fmax_r(-e * v_n_pre, 0.0f), fmax_r(v_n_pre, 0.0f));
  }
  __syncthreads();
  struct PairDesc {
    uint32_t i, j;
    float nx, ny, target;
  };
  const float w_l = w, w_sum = w + w;
  float2* const V_l = V;
  run_levels(nlev_c, m.lev_start,
             [&](uint32_t q) {
               const uint32_t k = m.lev_items[q];
               return PairDesc{m.act_i[k], m.act_j[k], m.act_w1[k], m.act_w2[k], m.act_t[k]};
             },
             [&](uint32_t, PairDesc d) {
               if (w_sum <= 0.0f) return;
               const V2 n_hat(d.nx, d.ny);
               float v_n_now = (V2(V_l[d.i]) - V2(V_l[d.j])).dot(n_hat);
               float dvn = d.target - v_n_now;
               float impulse = dvn / w_sum;
               V_l[d.i] = (V2(V_l[d.i]) + w_l * impulse * n_hat).f2();
               V_l[d.j] = (V2(V_l[d.j]) - w_l * impulse * n_hat).f2();
             });
  for (uint32_t k = na_p + tid(); k < na; k += nthr()) {
    const uint32_t i = m.act_i[k];
    m.act_flag[k] = 0;
    float dd;
    V2 n_hat;
    drum_sdf_world(U, V2(X[i]), U.to_local_next, U.to_world_next, dd, n_hat);
    V2 v_wall = wall_velocity(U.drum_omega, V2(X[i]) - r * n_hat);
    float v_n_pre = (V2(m.bvpre[i]) - v_wall).dot(n_hat);
    bool fresh = v_n_pre < -RESTITUTION_VELOCITY_THRESHOLD;
    if (fresh) {
      atomicAdd(&S.collisions, 1u);
      int bin = impact_energy_bin(0.5f * m.b_m * v_n_pre * v_n_pre);
      if (bin >= 0) atomicAdd(&S.hist[bin], 1u);
    }
    float e = fresh ? e_bw : 0.0f;
    if (-v_n_pre > impact_threshold) {
      V2 t_hat(-n_hat.y, n_hat.x);
      float slip = (V2(m.bvpre[i]) - v_wall).dot(t_hat) - r * m.bompre[i];
      m.act_rec[k] = MgImpactRecord{MG_IMPACT_BALL_WALL, i, MG_WALL_PARTNER, -v_n_pre, fabsf(slip), e};
      m.act_flag[k] = 1;
    }
    float target = fmax_r(fmax_r(-e * v_n_pre, 0.0f), fmax_r(v_n_pre, 0.0f));
    float v_n_now = (V2(V[i]) - v_wall).dot(n_hat);
    float dvn = target - v_n_now;
    if (w <= 0.0f) continue;
    V[i] = (V2(V[i]) + dvn * n_hat).f2();
  }
  __syncthreads();
}

// After the friction sweep, by warp 0: the wall work summed in wall-contact order, two adds per
// contact (dem.rs:870, 881), into S.fscal[1]; the active pair contacts counted; the restitution
// sweep's collision count and histogram cleared. Its own function, so that the unrolled shuffle
// loop is register-allocated apart from the DEM step around it.
static __device__ __noinline__ void friction_wall_work(const MillDev& m, uint32_t na, DemShared& S, StepOut& out) {
  if (tid() < 32) {
    const uint32_t lane = tid();
    float wall_work = 0.0f;
    uint32_t act = 0;
    for (uint32_t c = 0; c < na; c += 32) {
      uint32_t k = c + lane;
      bool wall = k < na && m.act_j[k] == NONE && m.act_bin[k] != -2;
      act += (k < na && m.act_j[k] != NONE) ? 1u : 0u;
      float a = wall ? m.act_w1[k] : 0.0f, b = wall ? m.act_w2[k] : 0.0f;
      const uint32_t mask = __ballot_sync(FULL, wall);
#pragma unroll
      for (int t = 0; t < 32; ++t) {
        const float at = __shfl_sync(FULL, a, t), bt = __shfl_sync(FULL, b, t);
        if ((mask >> t) & 1u) {
          wall_work += at;
          wall_work += bt;
        }
      }
    }
    act = warp_sum(act);
    if (lane == 0) {
      S.fscal[1] = wall_work;
      out.ctr.n_active_contacts = act;
      S.collisions = 0;
      for (int q = 0; q < MG_IMPACT_BINS; ++q) S.hist[q] = 0;
    }
  }
}

static __device__ __noinline__ void dem_step(const MillDev& m, const StepUniform& U, StepOut& out, MgImpactRecord* impacts,
                         uint32_t* err, DemShared& S, unsigned char* dsm) {
  const uint32_t n = m.nb;
  const float dt = U.dt;
  if (tid() == 0) { memset(&out.ds, 0, sizeof(out.ds)); out.n_impacts = 0; }
  __syncthreads();
  if (n == 0 || dt <= 0.0f) return;
  const float w = m.b_m > 0.0f ? 1.0f / m.b_m : 0.0f;
  const float w_rot = m.b_I > 0.0f ? 1.0f / m.b_I : 0.0f;
  const float r = m.b_r;
  const float impact_threshold = 0.1428f * sqrtf(-GRAVITY * 2.0f * r);
  const bool ext = U.dem_external != 0;
  // ball state: shared memory when it fits, global otherwise
  const bool staged = n <= m.smem_balls;
  float2 *X = m.bx, *V = m.bv;
  float *TH = m.bth, *OM = m.bom;
  if (staged) {
    X = reinterpret_cast<float2*>(dsm);
    V = X + n;
    TH = reinterpret_cast<float*>(V + n);
    OM = TH + n;
  }
  // step 0 sanitize, snapshots; step 1 predict (dem.rs:558-595)
  float max_disp = 0.0f, max_speed = 0.0f;
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 x(m.bx[i]), v(m.bv[i]);
    if (!x.finite() || !v.finite()) { x = V2(); v = V2(); }
    float th = m.bth[i], om = m.bom[i];
    m.bx0[i] = x.f2();
    m.bth0[i] = th;
    m.bvpre[i] = v.f2();
    m.bompre[i] = om;
    v.y += GRAVITY * dt;
    double cw = 0.0;
    if (ext) {
      double ke_before = 0.5 * (double)m.b_m * (double)v.len2() + 0.5 * (double)m.b_I * (double)(om * om);
      v += V2(m.imp[i]) * w;
      om += m.ang[i] * w_rot;
      double ke_after = 0.5 * (double)m.b_m * (double)v.len2() + 0.5 * (double)m.b_I * (double)(om * om);
      cw = ke_after - ke_before;
    }
    x += v * dt;
    X[i] = x.f2();
    V[i] = v.f2();
    OM[i] = om;
    TH[i] = th + om * dt;
    m.f_cw[i] = cw;
    max_disp = fmax_r(max_disp, v.len() * dt / fmax_r(2.0f * r, 1e-12f));
    max_speed = fmax_r(max_speed, v.len());
  }
  max_disp = block_max_f(max_disp);
  max_speed = block_max_f(max_speed);
  if (tid() < 32) {
    double cw = coupling_work_seq(m);
    float e = mech_energy_seq(m, X, V, OM);
    if (tid() == 0) { S.dscal[0] = cw; S.fscal[0] = e; }
  }
  __syncthreads();
  // step 2 broad phase (dem.rs:626-633)
  const uint32_t iters = U.dem_iterations > 1 ? U.dem_iterations : 1u;
  const float solve_margin = (float)iters * MAX_RECOVERY_FRACTION * 2.0f * r;
  const float cell = fmax_r(fmax_r(2.0f * r * 1.05f, 2.0f * r + max_speed * dt + solve_margin), 1e-6f);
  grid_build(X, n, cell, m.gBall, S.hg, err);
  uint32_t np = build_candidate_pairs(S.hg, m.gBall, m.pair_cnt, m.pair_i, m.pair_j, m.cap_pairs, err);
  if (tid() == 0) { S.npairs = np; out.ctr.n_ball_pairs = np; }
  __syncthreads();
  if (*err) return;
  np = S.npairs;
  // step 2.5 wall CCD (dem.rs:674-706)
  const float cap_depth = -MAX_RECOVERY_FRACTION * 2.0f * r;
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 x(X[i]), pl;
    // only the distance is used; interior balls are decided without the lifters
    const bool clear = x.finite() && drum_sdf_clear(U, rotate(x, U.to_local_next), r + cap_depth);
    float c_end = clear ? 0.0f : drum_sdf_world_dist(U, x, U.to_local_next, pl) - r;
    float t_hit = 1.0f;
    if (!clear && !(c_end >= cap_depth)) {
      float t;
      if (drum_toi_swept(U, V2(m.bx0[i]), x, U.drum_angle, U.drum_angle_next, r, t)) t_hit = fmin_r(1.0f, t);
    }
    if (t_hit < 1.0f) {
      atomicAdd(&out.ctr.ccd_clamps, 1u);
      V2 x0(m.bx0[i]);
      float path_len = (x - x0).len();
      float skin = CCD_SKIN_FRACTION * r;
      float t_skin = path_len > 1e-9f ? skin / path_len : 1.0f;
      float t_cl = fmin_r(t_hit + t_skin, 1.0f);
      X[i] = (x0 + (x - x0) * t_cl).f2();
    }
    m.lam_bw[i] = 0.0f;
  }
  for (uint32_t k = tid(); k < np; k += nthr()) m.lam_bb[k] = 0.0f;
  // step 3 projection: pairs in grid order, then walls, `iters` times (dem.rs:711-750).
  // A pair that stays apart never acts, so the sweep first runs only the pairs that start within
  // 2r + reach of touching (their relative order kept) plus every wall, while recording how far
  // each ball ever gets from its start position (the largest squared distance after any of its
  // moves). Afterwards every other pair must have stayed apart at all times: its start distance
  // less both balls' largest excursions exceeds 2r, with margins well above the f32 rounding of
  // the excursions and of the distance test. Otherwise the positions are restored and the sweep
  // runs again with the pairs it could not clear added. Either way the sweep's result is that of
  // the full order.
  const float reach = 0.25f * r;
  const float touch2 = (2.0f * r + reach) * (2.0f * r + reach);
  uint32_t* keep = reinterpret_cast<uint32_t*>(m.act_bin);  // pairs in the run (act_bin is free until step 5)
  for (uint32_t i = tid(); i < n; i += nthr()) m.bxs[i] = X[i];
  __syncthreads();
  for (uint32_t k = tid(); k < np; k += nthr())
    keep[k] = (V2(m.bxs[m.pair_i[k]]) - V2(m.bxs[m.pair_j[k]])).len2() < touch2 ? 1u : 0u;
  __syncthreads();
  stage_mark(out.stage, 15);
  uint32_t *lvl = m.dm_lvl, *di = m.act_i, *dj = m.act_j;
  float* dl = m.act_l;
  float* bm = m.bmove;  // per ball largest squared excursion of the run (shared memory when it fits)
  // One run: npi pair items (pair plist[q], or pair q when plist is null) by dependency levels in
  // warp 0, then the n walls of the iteration at once: in each iteration every wall comes after
  // every pair, and walls of different balls are independent.
  auto project = [&](uint32_t npi, const uint32_t* plist, bool track) {
    for (uint32_t k = tid(); k < npi; k += nthr()) { m.dm_pa[k] = NONE; m.dm_pb[k] = NONE; }
    // occurrence records: pair item q -> (i, 2q), (j, 2q+1)
    for (uint32_t q = tid(); q < 2 * npi; q += nthr()) {
      const uint32_t k = plist ? plist[q >> 1] : q >> 1;
      m.rec_i[q] = (q & 1u) ? m.pair_j[k] : m.pair_i[k];
    }
    for (uint32_t i = tid(); i < n; i += nthr()) m.lam_bw[i] = 0.0f;
    __syncthreads();
    preds_from_records(m.rec_i, 2 * npi, n, n, m.bk_start, m.bk_cur, m.bk_order, m.dm_pa, m.dm_pb,
                       [&](uint32_t q) { return q >> 1; }, [&](uint32_t q) { return q & 1u; });
    stage_mark(out.stage, 20);
    // sweep scratch (levels, level-ordered descriptors, multipliers): shared memory after the
    // ball state when the items fit, global otherwise
    lvl = m.dm_lvl; di = m.act_i; dj = m.act_j; dl = m.act_l;
    bm = m.bmove;
    if (staged) {
      const uint32_t used = (24u * n + 15u) & ~15u;
      const uint32_t fit = m.smem_bytes > used ? (m.smem_bytes - used) / 16u : 0u;
      if (npi <= fit) {
        lvl = reinterpret_cast<uint32_t*>(dsm + used);
        di = lvl + npi;
        dj = di + npi;
        dl = reinterpret_cast<float*>(dj + npi);
        // the excursions too when they fit: they are read and written level after level, and a
        // global store leaves the next level's read an L2 round trip
        const uint32_t off = used + 16u * npi;
        if (off + 4u * n <= m.smem_bytes) bm = reinterpret_cast<float*>(dsm + off);
      }
    }
    for (uint32_t i = tid(); i < n; i += nthr()) bm[i] = 0.0f;
    const uint32_t nlev = compute_levels(npi, m.dm_pa, m.dm_pb, lvl);
    stage_mark(out.stage, 21);
    bucket_levels(npi, lvl, nlev, m.lev_start, m.lev_cur, m.lev_items);
    // level-ordered sweep descriptors (the two balls) and a lambda accumulator
    for (uint32_t q = tid(); q < npi; q += nthr()) {
      const uint32_t k = m.lev_items[q];
      const uint32_t pk = plist ? plist[k] : k;
      di[q] = m.pair_i[pk];
      dj[q] = m.pair_j[pk];
      dl[q] = 0.0f;
    }
    __syncthreads();
    stage_mark(out.stage, 22);
    project_iterations(m, U, X, dl, bm, di, dj, nlev, iters, n, track, r, w, cap_depth);
    return npi;
  };
  // rounds: a failed check adds the pairs it could not clear and runs again from the start
  // positions; the last round runs every pair
  uint32_t ns = 0, nrun = 0;
  for (uint32_t round = 0;; ++round) {
    const bool all = round == PROJECTION_ROUNDS - 1;
    for (uint32_t k = tid(); k < np; k += nthr()) m.act_flag[k] = all ? 1u : keep[k];
    if (tid() == 0) m.act_flag[np] = 0;
    __syncthreads();
    ns = block_exclusive_scan(m.act_flag, np + 1);
    for (uint32_t k = tid(); k < np; k += nthr())
      if (m.act_flag[k + 1] != m.act_flag[k]) m.pr_list[m.act_flag[k]] = k;
    __syncthreads();
    nrun = project(ns, m.pr_list, ns < np);
    if (ns == np) break;
    // every pair left out stayed more than 2r apart (triangle inequality over the excursions)
    const double sep = 2.0 * (double)r * (1.0 + 1e-5);
    bool bad = false;
    for (uint32_t k = tid(); k < np; k += nthr()) {
      if (keep[k]) continue;
      const uint32_t i = m.pair_i[k], j = m.pair_j[k];
      const float2 a = m.bxs[i], b = m.bxs[j];
      const double dx = (double)a.x - (double)b.x, dy = (double)a.y - (double)b.y;
      const double ei = sqrt((double)bm[i]), ej = sqrt((double)bm[j]);
      const double slack = 1e-6 * (fabs((double)a.x) + fabs((double)a.y) + fabs((double)b.x) + fabs((double)b.y) + ei + ej);
      if (!(sqrt(dx * dx + dy * dy) - (ei + ej) * (1.0 + 1e-5) - slack >= sep)) { keep[k] = 1u; bad = true; }
    }
    if (!__syncthreads_or(bad)) break;
    for (uint32_t i = tid(); i < n; i += nthr()) X[i] = m.bxs[i];
    __syncthreads();
    stage_mark(out.stage, 39);
  }
  // the accumulated pair multipliers back to pair order (ContactBook, dem.rs:437-454; pairs left
  // out keep lambda 0, walls accumulated in lam_bw in place)
  for (uint32_t q = tid(); q < nrun; q += nthr()) m.lam_bb[m.pr_list[m.lev_items[q]]] = dl[q];
  __syncthreads();
  stage_mark(out.stage, 16);
  // step 4 velocity reconstruction (dem.rs:753-756)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V[i] = ((V2(X[i]) - V2(m.bx0[i])) / dt).f2();
    OM[i] = angle_diff(TH[i], m.bth0[i], err) / dt;
  }
  __syncthreads();
  // The contact sweeps visit only contacts with lambda_n > 0: pairs sorted by (i, j)
  // (dem.rs:459-467), then walls in ball order. The active pairs are compacted (ascending pair
  // index), bucketed by i (stable) and sorted by j inside a bucket (pairs are distinct, so j
  // decides): the order of sorting every pair and keeping the active ones.
  for (uint32_t k = tid(); k < np; k += nthr()) m.act_flag[k] = m.lam_bb[k] > 0.0f ? 1u : 0u;
  if (tid() == 0) m.act_flag[np] = 0;
  __syncthreads();
  const uint32_t na_p = block_exclusive_scan(m.act_flag, np + 1);  // active pair contacts
  for (uint32_t k = tid(); k < np; k += nthr()) {
    const uint32_t o = m.act_flag[k];
    if (m.act_flag[k + 1] != o) {
      m.pr_list[o] = k;
      m.dm_lvl[o] = m.pair_i[k];
    }
  }
  __syncthreads();
  block_bucket_sort(m.dm_lvl, na_p, n, m.bk_start, m.bk_cur, m.bk_order);
  for (uint32_t b = tid(); b < n; b += nthr()) {
    const uint32_t s = m.bk_start[b], e = m.bk_start[b + 1];
    if (e - s < 2u) continue;
    if (e - s <= 8u) {
      // up to 8 contacts: their keys (j) loaded once, a sorting network in registers (the keys
      // of one bucket are distinct, so any correct sort gives the insertion sort's order)
      const uint32_t c = e - s;
      uint32_t kv[8], vv[8];
#pragma unroll
      for (uint32_t t = 0; t < 8; ++t) {
        vv[t] = t < c ? m.bk_order[s + t] : 0u;
        kv[t] = t < c ? m.pair_j[m.pr_list[vv[t]]] : 0xFFFFFFFFu;
      }
      auto ce = [&](int i, int j) {
        if (kv[i] > kv[j]) {
          const uint32_t tk = kv[i], tv = vv[i];
          kv[i] = kv[j]; vv[i] = vv[j];
          kv[j] = tk; vv[j] = tv;
        }
      };
      ce(0, 1); ce(2, 3); ce(4, 5); ce(6, 7); ce(0, 2); ce(1, 3); ce(4, 6); ce(5, 7); ce(1, 2); ce(5, 6);
      ce(0, 4); ce(3, 7); ce(1, 5); ce(2, 6); ce(1, 4); ce(3, 6); ce(2, 4); ce(3, 5); ce(3, 4);
#pragma unroll
      for (uint32_t t = 0; t < 8; ++t)
        if (t < c) m.bk_order[s + t] = vv[t];
      continue;
    }
    for (uint32_t a = s + 1; a < e; ++a) {
      const uint32_t v = m.bk_order[a], vj = m.pair_j[m.pr_list[v]];
      uint32_t q = a;
      while (q > s && m.pair_j[m.pr_list[m.bk_order[q - 1]]] > vj) { m.bk_order[q] = m.bk_order[q - 1]; --q; }
      m.bk_order[q] = v;
    }
  }
  __syncthreads();
  for (uint32_t q = tid(); q < na_p; q += nthr()) {
    const uint32_t k = m.pr_list[m.bk_order[q]];
    m.act_i[q] = m.pair_i[k];
    m.act_j[q] = m.pair_j[k];
    m.act_l[q] = m.lam_bb[k];
  }
  for (uint32_t b = tid(); b < n; b += nthr()) m.act_flag[b] = m.lam_bw[b] > 0.0f ? 1u : 0u;
  if (tid() == 0) m.act_flag[n] = 0;
  __syncthreads();
  const uint32_t na = na_p + block_exclusive_scan(m.act_flag, n + 1);  // then the active walls
  for (uint32_t b = tid(); b < n; b += nthr()) {
    const uint32_t o = na_p + m.act_flag[b];
    if (na_p + m.act_flag[b + 1] == o) continue;
    m.act_i[o] = b;
    m.act_j[o] = NONE;
    m.act_l[o] = m.lam_bw[b];
  }
  __syncthreads();
  for (uint32_t k = tid(); k < na; k += nthr()) { m.dm_pa[k] = NONE; m.dm_pb[k] = NONE; }
  for (uint32_t q = tid(); q < 2 * na; q += nthr()) {
    uint32_t j = m.act_j[q >> 1];
    m.rec_i[q] = (q & 1u) ? (j == NONE ? n : j) : m.act_i[q >> 1];
  }
  __syncthreads();
  // buckets 0..n-1 are balls; bucket n collects the absent second ball of wall contacts
  preds_from_records(m.rec_i, 2 * na, n + 1, n, m.bk_start, m.bk_cur, m.bk_order, m.dm_pa, m.dm_pb,
                     [&](uint32_t q) { return q >> 1; }, [&](uint32_t q) { return q & 1u; });
  stage_mark(out.stage, 30);
  // step 5 friction (dem.rs:782-882)
  const MgMediaParams& md = U.media;
  // dependency levels of the active pair contacts, shared by the friction and restitution
  // sweeps: contacts of one level share no ball, so each level runs in parallel. Every wall
  // contact comes after every pair contact and touches one ball, so the walls then run at once.
  const uint32_t nlev_c = compute_levels(na_p, m.dm_pa, m.dm_pb, m.dm_lvl);
  bucket_levels(na_p, m.dm_lvl, nlev_c, m.lev_start, m.lev_cur, m.lev_items);
  stage_mark(out.stage, 38);
  friction_sweep(m, U, X, V, TH, OM, nlev_c, na_p, na, w, w_rot, r, dt);
  friction_wall_work(m, na, S, out);
  __syncthreads();
  stage_mark(out.stage, 17);
  // resync (dem.rs:887-890)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V[i] = ((V2(X[i]) - V2(m.bx0[i])) / dt).f2();
    OM[i] = angle_diff(TH[i], m.bth0[i], err) / dt;
  }
  __syncthreads();
  // step 6 restitution with impact accounting (dem.rs:909-1019); per-item records are compacted
  // in sweep order afterwards
  restitution_sweep(m, U, S, X, V, nlev_c, na_p, na, w, r, impact_threshold);
  if (tid() == 0) m.act_flag[na] = 0;
  __syncthreads();
  const uint32_t nrec = block_exclusive_scan(m.act_flag, na + 1);
  for (uint32_t k = tid(); k < na; k += nthr()) {
    uint32_t o = m.act_flag[k];
    if (m.act_flag[k + 1] != o && o < m.cap_impacts) impacts[o] = m.act_rec[k];
  }
  if (tid() == 0) {
    out.ds.collision_count = S.collisions;
    for (int q = 0; q < MG_IMPACT_BINS; ++q) out.ds.impact_energy_histogram[q] = S.hist[q];
    out.n_impacts = nrec;
    if (nrec > m.cap_impacts) atomicOr(err, ERR_IMPACTS);
  }
  // step 7 rolling resistance (dem.rs:1036-1055): per ball, sum lambda_n over its contacts in
  // sweep order (sorted pairs, then the wall); contacts with lambda_n <= 0 add +0 and are skipped
  if (md.rolling_friction > 0.0f && m.b_I > 0.0f) {
    for (uint32_t b = tid(); b < n; b += nthr()) {
      float tot = 0.0f;
      for (uint32_t q = m.bk_start[b]; q < m.bk_start[b + 1]; ++q) tot += fmax_r(m.act_l[m.bk_order[q] >> 1], 0.0f);
      float om = OM[b];
      if (tot <= 0.0f || om == 0.0f) continue;
      float normal_force = tot / dt;
      float max_dw = md.rolling_friction * normal_force * r / m.b_I * dt;
      float dw = fmin_r(max_dw, fabsf(om));
      OM[b] = om - (om < 0.0f ? -1.0f : 1.0f) * dw;
    }
  }
  __syncthreads();
  float e_final = 0.0f;
  if (tid() < 32) e_final = mech_energy_seq(m, X, V, OM);
  if (tid() == 0) {
    out.ds.wall_work_j = S.fscal[1];
    out.ds.dissipated_energy_j = S.fscal[0] + S.fscal[1] - e_final;
    out.ds.max_substep_displacement_over_diameter = max_disp;
    out.ds.coupling_work_j = (float)S.dscal[0];
  }
  if (staged) {
    for (uint32_t i = tid(); i < n; i += nthr()) {
      m.bx[i] = X[i];
      m.bv[i] = V[i];
      m.bth[i] = TH[i];
      m.bom[i] = OM[i];
    }
  }
  __syncthreads();
  stage_mark(out.stage, 18);
}

}  // namespace mg
