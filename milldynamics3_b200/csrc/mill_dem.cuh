// The ball half of the sub-step (DemState::step_recorded, dem.rs:530-1066) for one mill, executed
// by one thread block: per-ball stages in parallel; the broad phase materialises the candidate
// pairs in the grid's visiting order; the Gauss-Seidel projection, friction and restitution
// sweeps are replayed in the reference's order (bit-exact results).
#pragma once

#include "mill_geom.cuh"
#include "mill_grid.cuh"

namespace mg {

constexpr float RESTITUTION_VELOCITY_THRESHOLD = 0.02f;
constexpr float MAX_RECOVERY_FRACTION = 0.2f;
constexpr float CCD_SKIN_FRACTION = 1e-2f;

struct DemShared {
  GridHdr hg;
  uint32_t npairs;
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

// dem.rs:253-261 f32 mechanical energy, summed in ball order
__device__ float mech_energy_seq(const MillDev& m) {
  float e = 0.0f;
  for (uint32_t i = 0; i < m.nb; ++i) {
    e += 0.5f * m.b_m * V2(m.bv[i]).len2();
    e += 0.5f * m.b_I * m.bom[i] * m.bom[i];
    e += m.b_m * fabsf(GRAVITY) * m.bx[i].y;
  }
  return e;
}

__device__ void dem_step(const MillDev& m, const StepUniform& U, StepOut& out, MgImpactRecord* impacts,
                         uint32_t* err, DemShared& S) {
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
  float2 *X = m.bx, *V = m.bv;
  float *TH = m.bth, *OM = m.bom;
  // step 0 sanitize, snapshots; step 1 predict (dem.rs:558-595)
  float max_disp = 0.0f, max_speed = 0.0f;
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 x(X[i]), v(V[i]);
    if (!x.finite() || !v.finite()) { x = V2(); v = V2(); }
    m.bx0[i] = x.f2();
    m.bth0[i] = TH[i];
    m.bvpre[i] = v.f2();
    float om = OM[i];
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
    TH[i] = TH[i] + om * dt;
    m.f_cw[i] = cw;
    max_disp = fmax_r(max_disp, v.len() * dt / fmax_r(2.0f * r, 1e-12f));
    max_speed = fmax_r(max_speed, v.len());
  }
  max_disp = block_max_f(max_disp);
  max_speed = block_max_f(max_speed);
  if (tid() == 0) {
    double cw = 0.0;
    for (uint32_t i = 0; i < n; ++i) cw += m.f_cw[i];
    S.dscal[0] = cw;
    S.fscal[0] = mech_energy_seq(m);
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
    V2 x(X[i]);
    float d_end;
    V2 nn;
    drum_sdf_world(U, x, U.to_local_next, U.to_world_next, d_end, nn);
    float c_end = d_end - r;
    float t_hit = 1.0f;
    if (!(c_end >= cap_depth)) {
      float t;
      if (drum_toi_swept(U, V2(m.bx0[i]), x, U.drum_angle, U.drum_angle_next, r, t)) t_hit = fmin_r(1.0f, t);
    }
    if (t_hit < 1.0f) {
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
  __syncthreads();
  // step 3 projection: Gauss-Seidel over pairs in grid order, then walls (dem.rs:711-750)
  if (tid() == 0) {
    for (uint32_t it = 0; it < iters; ++it) {
      for (uint32_t k = 0; k < np; ++k) {
        uint32_t i = m.pair_i[k], j = m.pair_j[k];
        V2 xi(X[i]), xj(X[j]);
        V2 delta = xi - xj;
        float dist = delta.len();
        float c = dist - 2.0f * r;
        if (c >= 0.0f) continue;
        V2 n_hat = dist > 1e-9f ? delta / dist : V2(1.0f, 0.0f);
        float w_sum = w + w;
        if (w_sum <= 0.0f) continue;
        float c_eff = fmax_r(c, cap_depth);
        float d_lambda = -c_eff / w_sum;
        X[i] = (xi + w * d_lambda * n_hat).f2();
        X[j] = (xj - w * d_lambda * n_hat).f2();
        m.lam_bb[k] += d_lambda;
      }
      for (uint32_t i = 0; i < n; ++i) {
        V2 x(X[i]);
        float d;
        V2 n_hat;
        drum_sdf_world(U, x, U.to_local_next, U.to_world_next, d, n_hat);
        float c = d - r;
        if (c >= 0.0f) continue;
        if (w <= 0.0f) continue;
        float c_eff = fmax_r(c, cap_depth);
        float d_lambda = -c_eff / w;
        X[i] = (x + w * d_lambda * n_hat).f2();
        m.lam_bw[i] += d_lambda;
      }
    }
  }
  __syncthreads();
  // step 4 velocity reconstruction (dem.rs:753-756)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V[i] = ((V2(X[i]) - V2(m.bx0[i])) / dt).f2();
    OM[i] = angle_diff(TH[i], m.bth0[i], err) / dt;
  }
  __syncthreads();
  // contacts sorted by (i, j) (dem.rs:459-467): bucket by i (stable), then by j inside a bucket
  block_bucket_sort(m.pair_i, np, n, m.bk_start, m.bk_cur, m.bk_order);
  for (uint32_t b = tid(); b < n; b += nthr()) {
    uint32_t s = m.bk_start[b], e = m.bk_start[b + 1];
    for (uint32_t a = s + 1; a < e; ++a) {
      uint32_t v = m.bk_order[a];
      uint32_t vj = m.pair_j[v];
      uint32_t q = a;
      while (q > s && m.pair_j[m.bk_order[q - 1]] > vj) { m.bk_order[q] = m.bk_order[q - 1]; --q; }
      m.bk_order[q] = v;
    }
  }
  __syncthreads();
  for (uint32_t q = tid(); q < np; q += nthr()) {
    uint32_t k = m.bk_order[q];
    m.cs_i[q] = m.pair_i[k];
    m.cs_j[q] = m.pair_j[k];
    m.cs_l[q] = m.lam_bb[k];
  }
  __syncthreads();
  // step 5 friction: sorted pairs, then walls (dem.rs:782-882)
  const MgMediaParams& md = U.media;
  if (tid() == 0) {
    uint32_t act = 0;
    for (uint32_t q = 0; q < np; ++q) {
      float lambda_n = m.cs_l[q];
      if (lambda_n <= 0.0f) continue;
      ++act;
      uint32_t i = m.cs_i[q], j = m.cs_j[q];
      V2 delta = V2(X[i]) - V2(X[j]);
      float dist = delta.len();
      V2 n_hat = dist > 1e-9f ? delta / dist : V2(1.0f, 0.0f);
      V2 t_hat(-n_hat.y, n_hat.x);
      float v_t = (V2(V[i]) - V2(V[j])).dot(t_hat) - r * OM[i] - r * OM[j];
      float w_sum_t = w + w + r * r * w_rot + r * r * w_rot;
      if (w_sum_t <= 0.0f) continue;
      float raw = -v_t * dt / w_sum_t;
      float mu = effective_friction(md.friction_ball_ball, md.friction_ball_ball_static, v_t, md.friction_velocity_scale_m_s);
      float max_mag = mu * lambda_n;
      float dlt = clamp_r(raw, -max_mag, max_mag);
      X[i] = (V2(X[i]) + w * dlt * t_hat).f2();
      X[j] = (V2(X[j]) - w * dlt * t_hat).f2();
      TH[i] -= r * w_rot * dlt;
      TH[j] -= r * w_rot * dlt;
      V2 dv = w * dlt * t_hat / dt;
      float domega = -r * w_rot * dlt / dt;
      V[i] = (V2(V[i]) + dv).f2();
      V[j] = (V2(V[j]) - dv).f2();
      OM[i] += domega;
      OM[j] += domega;
    }
    out.ctr.n_active_contacts = act;
    float wall_work = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
      float lambda_n = m.lam_bw[i];
      if (lambda_n <= 0.0f) continue;
      float dd;
      V2 n_hat;
      drum_sdf_world(U, V2(X[i]), U.to_local_next, U.to_world_next, dd, n_hat);
      V2 t_hat(-n_hat.y, n_hat.x);
      V2 v_wall = wall_velocity(U.drum_omega, V2(X[i]) - r * n_hat);
      float v_t = (V2(V[i]) - v_wall).dot(t_hat) - r * OM[i];
      float w_sum_t = w + r * r * w_rot;
      if (w_sum_t <= 0.0f) continue;
      float raw = -v_t * dt / w_sum_t;
      float mu = effective_friction(md.friction_ball_wall, md.friction_ball_wall_static, v_t, md.friction_velocity_scale_m_s);
      float max_mag = mu * lambda_n;
      float dlt = clamp_r(raw, -max_mag, max_mag);
      X[i] = (V2(X[i]) + w * dlt * t_hat).f2();
      TH[i] -= r * w_rot * dlt;
      V[i] = (V2(V[i]) + w * dlt * t_hat / dt).f2();
      OM[i] += -r * w_rot * dlt / dt;
      wall_work += (dlt / dt) * t_hat.dot(v_wall);
      wall_work += (lambda_n / dt) * n_hat.dot(v_wall);
    }
    S.fscal[1] = wall_work;
  }
  __syncthreads();
  // resync (dem.rs:887-890)
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V[i] = ((V2(X[i]) - V2(m.bx0[i])) / dt).f2();
    OM[i] = angle_diff(TH[i], m.bth0[i], err) / dt;
  }
  __syncthreads();
  // step 6 restitution with impact accounting (dem.rs:909-1019)
  if (tid() == 0) {
    uint32_t collisions = 0, nrec = 0;
    uint32_t hist[MG_IMPACT_BINS];
    for (int k = 0; k < MG_IMPACT_BINS; ++k) hist[k] = 0;
    for (uint32_t q = 0; q < np; ++q) {
      if (m.cs_l[q] <= 0.0f) continue;
      uint32_t i = m.cs_i[q], j = m.cs_j[q];
      V2 delta = V2(X[i]) - V2(X[j]);
      float dist = delta.len();
      V2 n_hat = dist > 1e-9f ? delta / dist : V2(1.0f, 0.0f);
      float v_n_pre = (V2(m.bvpre[i]) - V2(m.bvpre[j])).dot(n_hat);
      bool fresh = v_n_pre < -RESTITUTION_VELOCITY_THRESHOLD;
      if (fresh) {
        collisions += 1;
        int bin = impact_energy_bin(0.5f * (m.b_m * 0.5f) * v_n_pre * v_n_pre);
        if (bin >= 0) hist[bin] += 1;
      }
      float e = fresh ? md.restitution_ball_ball : 0.0f;
      if (-v_n_pre > impact_threshold) {
        if (nrec < m.cap_impacts) {
          V2 t_hat(-n_hat.y, n_hat.x);
          float slip = (V2(m.bvpre[i]) - V2(m.bvpre[j])).dot(t_hat) - r * m.bompre[i] - r * m.bompre[j];
          impacts[nrec] = MgImpactRecord{MG_IMPACT_BALL_BALL, i, j, -v_n_pre, fabsf(slip), e};
        }
        ++nrec;
      }
      float target = fmax_r(fmax_r(-e * v_n_pre, 0.0f), fmax_r(v_n_pre, 0.0f));
      float v_n_now = (V2(V[i]) - V2(V[j])).dot(n_hat);
      float dvn = target - v_n_now;
      float w_sum = w + w;
      if (w_sum <= 0.0f) continue;
      float impulse = dvn / w_sum;
      V[i] = (V2(V[i]) + w * impulse * n_hat).f2();
      V[j] = (V2(V[j]) - w * impulse * n_hat).f2();
    }
    for (uint32_t i = 0; i < n; ++i) {
      float lambda_n = m.lam_bw[i];
      if (lambda_n <= 0.0f) continue;
      float dd;
      V2 n_hat;
      drum_sdf_world(U, V2(X[i]), U.to_local_next, U.to_world_next, dd, n_hat);
      V2 v_wall = wall_velocity(U.drum_omega, V2(X[i]) - r * n_hat);
      float v_n_pre = (V2(m.bvpre[i]) - v_wall).dot(n_hat);
      bool fresh = v_n_pre < -RESTITUTION_VELOCITY_THRESHOLD;
      if (fresh) {
        collisions += 1;
        int bin = impact_energy_bin(0.5f * m.b_m * v_n_pre * v_n_pre);
        if (bin >= 0) hist[bin] += 1;
      }
      float e = fresh ? md.restitution_ball_wall : 0.0f;
      if (-v_n_pre > impact_threshold) {
        if (nrec < m.cap_impacts) {
          V2 t_hat(-n_hat.y, n_hat.x);
          float slip = (V2(m.bvpre[i]) - v_wall).dot(t_hat) - r * m.bompre[i];
          impacts[nrec] = MgImpactRecord{MG_IMPACT_BALL_WALL, i, MG_WALL_PARTNER, -v_n_pre, fabsf(slip), e};
        }
        ++nrec;
      }
      float target = fmax_r(fmax_r(-e * v_n_pre, 0.0f), fmax_r(v_n_pre, 0.0f));
      float v_n_now = (V2(V[i]) - v_wall).dot(n_hat);
      float dvn = target - v_n_now;
      if (w <= 0.0f) continue;
      V[i] = (V2(V[i]) + dvn * n_hat).f2();
    }
    out.ds.collision_count = collisions;
    for (int k = 0; k < MG_IMPACT_BINS; ++k) out.ds.impact_energy_histogram[k] = hist[k];
    out.n_impacts = nrec;
    if (nrec > m.cap_impacts) atomicOr(err, ERR_IMPACTS);
    // step 7 rolling resistance sums, in sorted-contact order then walls (dem.rs:1036-1044)
    if (md.rolling_friction > 0.0f && m.b_I > 0.0f) {
      for (uint32_t i = 0; i < n; ++i) m.lam_tot[i] = 0.0f;
      for (uint32_t q = 0; q < np; ++q) {
        float l = fmax_r(m.cs_l[q], 0.0f);
        m.lam_tot[m.cs_i[q]] += l;
        m.lam_tot[m.cs_j[q]] += l;
      }
      for (uint32_t i = 0; i < n; ++i) m.lam_tot[i] += fmax_r(m.lam_bw[i], 0.0f);
    }
  }
  __syncthreads();
  if (md.rolling_friction > 0.0f && m.b_I > 0.0f) {
    for (uint32_t i = tid(); i < n; i += nthr()) {
      float ln = m.lam_tot[i];
      float om = OM[i];
      if (ln <= 0.0f || om == 0.0f) continue;
      float normal_force = ln / dt;
      float max_dw = md.rolling_friction * normal_force * r / m.b_I * dt;
      float dw = fmin_r(max_dw, fabsf(om));
      OM[i] = om - (om < 0.0f ? -1.0f : 1.0f) * dw;
    }
  }
  __syncthreads();
  if (tid() == 0) {
    float e_final = mech_energy_seq(m);
    out.ds.wall_work_j = S.fscal[1];
    out.ds.dissipated_energy_j = S.fscal[0] + S.fscal[1] - e_final;
    out.ds.max_substep_displacement_over_diameter = max_disp;
    out.ds.coupling_work_j = (float)S.dscal[0];
  }
  __syncthreads();
}

}  // namespace mg
