// The impact-energy accumulator (stress.rs:110-171, StressAccum::update) on the device: after
// each sub-step the mill's impact records are folded, in record order, into the f64 EMA rates,
// the 28-bin log histogram and the cumulative sums. The reference's debounce map (the time each
// (ball, partner) pair was last counted, BTreeMap<(u32, u32), f64>) is an open-addressing table
// in device memory. Only whether a key was counted within the window decides anything, so a slot
// whose time lies a window or more in the past is free for another key (the reference's periodic
// pruning of old entries changes no decision either); keys are never removed, so a key's probe
// sequence from its hash never crosses an empty slot and a key is never stored twice.
#pragma once

#include "mill_common.cuh"

namespace mg {

// The first slot of key k's probe sequence (host and device: a table carried to a new arena is
// re-filled on the host with the same hash).
MG_HD uint32_t stress_slot(uint2 k, uint32_t mask) {
  unsigned long long z = ((unsigned long long)k.x << 32) | (unsigned long long)k.y;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return (uint32_t)(z ^ (z >> 31)) & mask;
}

// Whether the impact of key k counts at now_s (and records it when it does). False: counted
// within the window. Sets ERR_STRESS (and counts it) when no slot is free.
__device__ __forceinline__ bool stress_counts(const MillDev& m, uint2 k, double now_s, double window, uint32_t* err) {
  const uint32_t mask = m.st_cap - 1u;
  uint32_t slot = stress_slot(k, mask), reuse = NONE;
  for (uint32_t probe = 0; probe < m.st_cap; ++probe, slot = (slot + 1u) & mask) {
    const uint2 s = m.st_key[slot];
    if (s.x == k.x && s.y == k.y) {
      if (now_s - m.st_time[slot] < window) return false;
      m.st_time[slot] = now_s;
      return true;
    }
    if (s.x == 0u && s.y == 0u) {
      const uint32_t at = reuse != NONE ? reuse : slot;
      m.st_key[at] = k;
      m.st_time[at] = now_s;
      return true;
    }
    if (reuse == NONE && !(now_s - m.st_time[slot] < window)) reuse = slot;
  }
  if (reuse != NONE) {
    m.st_key[reuse] = k;
    m.st_time[reuse] = now_s;
  } else {
    atomicOr(err, ERR_STRESS);
  }
  return true;
}

// stress.rs:59-64 se_bin
__device__ __forceinline__ int stress_se_bin(double e_hat) {
  if (isnan(e_hat) || e_hat <= 0.0) return 0;
  double t = (log10(e_hat) + 3.0) * 4.0;
  if (!(t > 0.0)) t = 0.0;
  if (t >= 27.0) return 27;
  return (int)t;
}

// StressAccum::update for one sub-step's records (one thread; the sums are in record order):
// m3 = disc mass * 4/3 r, scale m3 g d, window DEBOUNCE_FACTOR sqrt(d / g) (stress.rs:49, lib.rs
// update_grinding_stats), EMA weight alpha over sub_dt, wall work of the sub-step.
__device__ inline void stress_update(const MillDev& m, const MgImpactRecord* recs, uint32_t n, double now_s,
                                     double sub_dt, double alpha, double wall_work_j, uint32_t* err) {
  const double THR[6] = {0.03, 0.1, 0.3, 1.0, 3.0, 10.0};
  const double r = (double)m.b_r;
  const double m3 = (double)m.b_m * 4.0 / 3.0 * r;
  const double d = 2.0 * r;
  const double scale_j = m3 * 9.81 * d;
  const double window = 0.25 * sqrt(d / 9.81);
  StressState& st = *m.stress;
  st.updates += 1;
  double count[4] = {0.0, 0.0, 0.0, 0.0}, se_hat[4] = {0.0, 0.0, 0.0, 0.0};
  double hist[MG_SE_BINS], above[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < MG_SE_BINS; ++b) hist[b] = 0.0;
  for (uint32_t q = 0; q < n; ++q) {
    const MgImpactRecord rec = recs[q];
    if (window > 0.0) {
      uint2 key = rec.partner == MG_WALL_PARTNER ? make_uint2(rec.ball, MG_WALL_PARTNER)
                                                 : make_uint2(min(rec.ball, rec.partner), max(rec.ball, rec.partner));
      if (!stress_counts(m, key, now_s, window, err)) continue;
    }
    const bool bb = rec.kind == MG_IMPACT_BALL_BALL;
    const double vn = rec.normal_speed, vs = rec.slip_speed;
    const int cls = bb ? (vs > vn ? 1 : 0) : (vs > vn ? 3 : 2);
    const double m_red = bb ? 0.5 * m3 : m3;
    const double se = 0.5 * m_red * (vn * vn + vs * vs);
    const double e_hat = se / scale_j;
    count[cls] += 1.0;
    se_hat[cls] += e_hat;
    hist[stress_se_bin(e_hat)] += 1.0;
    for (int t = 0; t < 6; ++t)
      if (e_hat >= THR[t]) above[t] += se;
  }
  st.cum_wall_j += wall_work_j;
  for (int t = 0; t < 6; ++t) st.cum_above_j[t] += above[t];
  for (int c = 0; c < 4; ++c) {
    st.count_rate[c] += alpha * (count[c] / sub_dt - st.count_rate[c]);
    st.se_hat_rate[c] += alpha * (se_hat[c] / sub_dt - st.se_hat_rate[c]);
  }
  for (int b = 0; b < MG_SE_BINS; ++b) st.hist_rate[b] += alpha * (hist[b] / sub_dt - st.hist_rate[b]);
  for (int t = 0; t < 6; ++t) st.above_rate_j[t] += alpha * (above[t] / sub_dt - st.above_rate_j[t]);
}

}  // namespace mg
