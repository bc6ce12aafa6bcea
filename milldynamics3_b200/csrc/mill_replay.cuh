// Exact parallel replay of the reference's Gauss-Seidel sweeps.
//
// A sweep is a sequence of items; each item touches at most two balls (a ball-ball contact or a
// ball-wall contact). Executing any two items that share no ball in either order gives the same
// floating-point results, so the sequential result is reproduced exactly by any schedule that
// keeps, for every ball, the items touching it in sequence order. pred_a[k] / pred_b[k] name the
// previous item touching each of item k's balls (NONE when there is none).
//
//   * level replay: level(k) = 1 + max(level(preds)); all items of one level are independent and
//     run in parallel, levels in increasing order (used for the long projection sweeps);
//   * chunked replay: one warp walks the sequence 32 items at a time and runs, round by round,
//     the items whose in-chunk predecessors are done (used for the short contact sweeps).
#pragma once

#include "mill_block.cuh"

namespace mg {

constexpr uint32_t FULL = 0xffffffffu;

// Records r in [0, nrec) name a (ball key[r], item item_of(r)) occurrence, numbered so that
// records of earlier items come first. Bucket-sorts them by key into nbk buckets (stable) and,
// for the first nballs buckets, stores for each record the item of the previous record of the
// same ball into pred_a / pred_b (per slot_of(r)). Buckets from nballs on collect placeholders.
template <class ItemOf, class SlotOf>
__device__ void preds_from_records(const uint32_t* key, uint32_t nrec, uint32_t nbk, uint32_t nballs, uint32_t* start,
                                   uint32_t* cur, uint32_t* order, uint32_t* pred_a, uint32_t* pred_b, ItemOf item_of,
                                   SlotOf slot_of) {
  block_bucket_sort(key, nrec, nbk, start, cur, order);
  for (uint32_t b = tid(); b < nballs; b += nthr()) {
    uint32_t prev = NONE;
    for (uint32_t q = start[b]; q < start[b + 1]; ++q) {
      uint32_t r = order[q];
      uint32_t it = item_of(r);
      if (slot_of(r)) pred_b[it] = prev;
      else pred_a[it] = prev;
      prev = it;
    }
  }
  __syncthreads();
}

// Levels of items [0, n) (warp 0; chunks of 32 items, in-chunk propagation by shuffles).
// Returns the number of levels (block-uniform).
static __device__ uint32_t compute_levels(uint32_t n, const uint32_t* pred_a, const uint32_t* pred_b, uint32_t* lvl) {
  __shared__ uint32_t nlev;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    uint32_t maxl = 0;
    // the next chunk's predecessors are loaded while this chunk propagates
    uint32_t a_next = (uint32_t)lane < n ? pred_a[lane] : NONE, b_next = (uint32_t)lane < n ? pred_b[lane] : NONE;
    for (uint32_t c = 0; c < n; c += 32) {
      uint32_t k = c + lane;
      const uint32_t a = a_next, b = b_next;
      const uint32_t kn = k + 32;
      a_next = kn < n ? pred_a[kn] : NONE;
      b_next = kn < n ? pred_b[kn] : NONE;
      int base = 0, la = -1, lb = -1;
      if (k < n) {
        if (a != NONE) { if (a >= c) la = (int)(a - c); else base = max(base, (int)lvl[a] + 1); }
        if (b != NONE) { if (b >= c) lb = (int)(b - c); else base = max(base, (int)lvl[b] + 1); }
      }
      int L = base;
      for (int round = 0; round < 33; ++round) {
        int A = __shfl_sync(FULL, L, la < 0 ? lane : la) + 1;
        int Bv = __shfl_sync(FULL, L, lb < 0 ? lane : lb) + 1;
        int nl = base;
        if (la >= 0) nl = max(nl, A);
        if (lb >= 0) nl = max(nl, Bv);
        bool changed = nl != L;
        L = nl;
        if (!__any_sync(FULL, changed)) break;
      }
      if (k < n) { lvl[k] = (uint32_t)L; maxl = max(maxl, (uint32_t)L + 1); }
      __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) maxl = max(maxl, __shfl_xor_sync(FULL, maxl, o));
    if (lane == 0) nlev = maxl;
  }
  __syncthreads();
  uint32_t r = nlev;
  __syncthreads();
  return r;
}

// Groups items by level: lev_start[0..nlev], lev_items[] (order inside a level is irrelevant).
static __device__ void bucket_levels(uint32_t n, const uint32_t* lvl, uint32_t nlev, uint32_t* lev_start, uint32_t* lev_cur,
                              uint32_t* lev_items) {
  for (uint32_t l = tid(); l <= nlev; l += nthr()) lev_start[l] = 0;
  __syncthreads();
  for (uint32_t k = tid(); k < n; k += nthr()) atomicAdd(&lev_start[lvl[k]], 1u);
  __syncthreads();
  block_exclusive_scan(lev_start, nlev + 1);
  for (uint32_t l = tid(); l < nlev; l += nthr()) lev_cur[l] = lev_start[l];
  __syncthreads();
  for (uint32_t k = tid(); k < n; k += nthr()) lev_items[atomicAdd(&lev_cur[lvl[k]], 1u)] = k;
  __syncthreads();
}

// Runs exec(q, load(q)) for every level-ordered position q, level by level, in warp 0; the block
// waits at the end. Positions [lev_start[l], lev_start[l+1]) form level l. load(q) must read only
// what the levels do not write (the item's descriptor).
template <class Load, class Exec>
__device__ void run_levels(uint32_t nlev, const uint32_t* lev_start, Load load, Exec exec) {
  if (threadIdx.x < 32 && nlev > 0) {
    const uint32_t lane = threadIdx.x;
    // level t is [s, e); its first descriptor per lane and the next level's end are fetched one
    // level ahead, so only the item's own dependent loads sit between two levels
    uint32_t e = lev_start[1];
    uint32_t q = lev_start[0] + lane;
    auto d = q < e ? load(q) : decltype(load(0u)){};
    for (uint32_t t = 0; t < nlev; ++t) {
      const uint32_t e_next = t + 1 < nlev ? lev_start[t + 2] : e;
      const uint32_t qn = e + lane;
      const auto dn = qn < e_next ? load(qn) : decltype(load(0u)){};
      if (q < e) exec(q, d);
      for (uint32_t q2 = q + 32; q2 < e; q2 += 32) exec(q2, load(q2));  // levels wider than a warp
      __syncwarp();
      e = e_next;
      q = qn;
      d = dn;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- per-ball sweeps over fluid
// The drag and buoyancy sweeps (pbf.rs:1824-2011, 2042-2121) visit balls in index order; ball b
// reads and writes the velocities of its items (fluid particles), so it depends on the earlier
// balls that share an item. Balls are claimed in index order by the warps of the block, and a
// warp starts ball b once every earlier ball sharing one of b's items is done.

__shared__ uint32_t g_ticket;

// Packs the per-ball item lists (item_j[b * cap + s], s < cnt[b]) into records in ball order:
// rec_off[0..nb], rec_key[r] = fluid index, rec_ball[r] = ball. Returns the record count.
static __device__ uint32_t pack_ball_items(const uint32_t* item_j, const uint32_t* cnt, uint32_t cap, uint32_t nb,
                                    uint32_t* rec_off, uint32_t* rec_key, uint32_t* rec_ball) {
  for (uint32_t b = tid(); b < nb; b += nthr()) rec_off[b] = cnt[b];
  if (tid() == 0) rec_off[nb] = 0;
  __syncthreads();
  uint32_t total = block_exclusive_scan(rec_off, nb + 1);
  for (uint32_t b = tid() >> 5; b < nb; b += nthr() >> 5) {
    const uint32_t o = rec_off[b], c = cnt[b];
    for (uint32_t s = tid() & 31u; s < c; s += 32) { rec_key[o + s] = item_j[(size_t)b * cap + s]; rec_ball[o + s] = b; }
  }
  __syncthreads();
  return total;
}

// rec_pred[r] = the ball of the previous record with the same fluid index (NONE if first).
static __device__ void ball_item_preds(const uint32_t* rec_key, const uint32_t* rec_ball, uint32_t nrec, uint32_t nf,
                                uint32_t* start, uint32_t* cur, uint32_t* order, uint32_t* rec_pred) {
  block_bucket_sort(rec_key, nrec, nf, start, cur, order);
  for (uint32_t j = tid(); j < nf; j += nthr()) {
    uint32_t prev = NONE;
    for (uint32_t q = start[j]; q < start[j + 1]; ++q) {
      uint32_t r = order[q];
      rec_pred[r] = prev;
      prev = rec_ball[r];
    }
  }
  __syncthreads();
}


// Runs fn(b, lane) once per ball, one warp per ball, in a dependency-respecting order. done[] is
// nb words of scratch (shared or global). Waits are bounded: a wait that runs out sets
// ERR_BUDGET in *err and lets the ball proceed.
// Each ball runs in three parts: st = pre(b, lane) before the wait (loads and everything that
// does not read what the sweep writes), run(b, lane, st) once the earlier balls sharing an item
// are done (the part that reads and writes the swept velocities), then, after b is flagged done,
// post(b, lane, st) (per-ball outputs that no other ball reads during the sweep). Only run() lies
// on the dependency chain.
// acct (optional, 3 counters): clock cycles summed over balls spent in pre, waiting, and in
// run + post.
// Warp-uniform wait until every lane's ball p (NONE: no wait) is flagged done: the lanes poll
// together and sleep together, so the warp never diverges here (lanes that spun on their own
// were measured to leave the shuffle-heavy code after the wait several times slower).
__device__ __forceinline__ void wait_ball_done(volatile uint32_t* vdone, uint32_t p, uint32_t spin_ns,
                                               uint32_t spin_limit, uint32_t* err) {
  for (uint32_t spins = 0;; ++spins) {
    const bool ok = p == NONE || vdone[p] != 0u;
    if (__all_sync(FULL, ok)) break;
    if (spins > spin_limit) {
      if ((threadIdx.x & 31u) == 0) atomicOr(err, ERR_BUDGET);
      break;
    }
    __nanosleep(spin_ns);  // yield issue slots to the warps on the critical path
  }
}

// Warps from `warps` on sit the sweep out (they wait at the closing barrier). A wait gives up after
// spin_limit polls. skip_done names a ball whose done flag is never set (tests of the bounded
// wait only; NONE otherwise).
template <class Pre, class Run, class Post>
__device__ void ball_dataflow(uint32_t nb, const uint32_t* rec_off, const uint32_t* rec_pred, uint32_t* done,
                              uint32_t warps, uint32_t spin_ns, uint32_t spin_limit, uint32_t skip_done, uint32_t* err,
                              unsigned long long* acct, Pre pre, Run run, Post post) {
  for (uint32_t b = tid(); b < nb; b += nthr()) done[b] = 0u;
  if (tid() == 0) g_ticket = 0;
  __syncthreads();
  volatile uint32_t* vdone = done;
  const int lane = threadIdx.x & 31;
  unsigned long long t_pre = 0, t_wait = 0, t_run = 0;
  for (;;) {
    if ((threadIdx.x >> 5) >= warps) break;
    uint32_t b = 0;
    if (lane == 0) b = atomicAdd(&g_ticket, 1u);
    b = __shfl_sync(FULL, b, 0);
    if (b >= nb) break;
    const long long t0 = clock64();
    const uint32_t r0 = rec_off[b], r1 = rec_off[b + 1];
    const uint32_t p0 = r0 + lane < r1 ? rec_pred[r0 + lane] : NONE;
    auto st = pre(b, lane);
    const long long t1 = clock64();
    wait_ball_done(vdone, p0, spin_ns, spin_limit, err);
    for (uint32_t c = r0 + 32; c < r1; c += 32)
      wait_ball_done(vdone, c + lane < r1 ? rec_pred[c + lane] : NONE, spin_ns, spin_limit, err);
    __syncwarp();
    __threadfence_block();
    const long long t2 = clock64();
    run(b, lane, st);
    __threadfence_block();
    __syncwarp();
    if (lane == 0 && b != skip_done) vdone[b] = 1u;
    post(b, lane, st);
    t_pre += (unsigned long long)(t1 - t0);
    t_wait += (unsigned long long)(t2 - t1);
    t_run += (unsigned long long)(clock64() - t2);
  }
  if (acct && lane == 0 && (t_pre | t_wait | t_run)) {
    atomicAdd(&acct[0], t_pre);
    atomicAdd(&acct[1], t_wait);
    atomicAdd(&acct[2], t_run);
  }
  __syncthreads();
}

// Three in-order sums over the lanes' values t = 0..lim-1, added to a, b, c (the same on every
// lane): the lanes store their values to the warp's shared scratch and lane 0 adds them in lane
// order (independent loads, three interleaved chains of additions), then broadcasts the sums.
__shared__ float g_seq_buf[MAX_BLOCK_WARPS][3][32];
__device__ __forceinline__ void lane_seq_sum3(float& a, float& b, float& c, float va, float vb, float vc,
                                              uint32_t lim) {
  const uint32_t lane = threadIdx.x & 31u;
  float(*B)[32] = g_seq_buf[threadIdx.x >> 5];
  B[0][lane] = va;
  B[1][lane] = vb;
  B[2][lane] = vc;
  __syncwarp();
  if (lane == 0) {
    // four terms' loads ahead of their additions
    uint32_t t = 0;
    for (; t + 4 <= lim; t += 4) {
      const float a0 = B[0][t], a1 = B[0][t + 1], a2 = B[0][t + 2], a3 = B[0][t + 3];
      const float b0 = B[1][t], b1 = B[1][t + 1], b2 = B[1][t + 2], b3 = B[1][t + 3];
      const float c0 = B[2][t], c1 = B[2][t + 1], c2 = B[2][t + 2], c3 = B[2][t + 3];
      a += a0; b += b0; c += c0;
      a += a1; b += b1; c += c1;
      a += a2; b += b2; c += c2;
      a += a3; b += b3; c += c3;
    }
    for (; t < lim; ++t) {
      a += B[0][t];
      b += B[1][t];
      c += B[2][t];
    }
  }
  __syncwarp();
  a = __shfl_sync(FULL, a, 0);
  b = __shfl_sync(FULL, b, 0);
  c = __shfl_sync(FULL, c, 0);
}

// Block-wide in-order f32 sum init + term(0) + term(1) + ... + term(n-1), every term added (the
// reference's sequential f32 accumulations): all threads evaluate a chunk of terms into shared
// memory (the warps' scratch above, free outside the per-ball sweeps), then thread 0 adds them in
// order with the loads running ahead of the additions. All threads call it; all get the result.
// With SKIP_NONFINITE, non-finite terms are left out (not added).
template <bool SKIP_NONFINITE = false, class Term>
__device__ float block_seq_sum_f32(float init, uint32_t n, Term term) {
  constexpr uint32_t CHUNK = MAX_BLOCK_WARPS * 3 * 32;
  float* buf = &g_seq_buf[0][0][0];
  __shared__ float res;
  float acc = init;
  for (uint32_t c0 = 0; c0 < n; c0 += CHUNK) {
    const uint32_t cnt = min(CHUNK, n - c0);
    for (uint32_t k = tid(); k < cnt; k += nthr()) buf[k] = term(c0 + k);
    __syncthreads();
    if (tid() == 0) {
      uint32_t k = 0;
      for (; k + 8 <= cnt; k += 8) {
        const float x0 = buf[k], x1 = buf[k + 1], x2 = buf[k + 2], x3 = buf[k + 3];
        const float x4 = buf[k + 4], x5 = buf[k + 5], x6 = buf[k + 6], x7 = buf[k + 7];
        if (!SKIP_NONFINITE || finite_f(x0)) acc += x0;
        if (!SKIP_NONFINITE || finite_f(x1)) acc += x1;
        if (!SKIP_NONFINITE || finite_f(x2)) acc += x2;
        if (!SKIP_NONFINITE || finite_f(x3)) acc += x3;
        if (!SKIP_NONFINITE || finite_f(x4)) acc += x4;
        if (!SKIP_NONFINITE || finite_f(x5)) acc += x5;
        if (!SKIP_NONFINITE || finite_f(x6)) acc += x6;
        if (!SKIP_NONFINITE || finite_f(x7)) acc += x7;
      }
      for (; k < cnt; ++k)
        if (!SKIP_NONFINITE || finite_f(buf[k])) acc += buf[k];
    }
    __syncthreads();
  }
  if (tid() == 0) res = acc;
  __syncthreads();
  const float r = res;
  __syncthreads();
  return r;
}

// In-order sum over the lanes' values t = 0..lim-1 (every lane computes the same chain).
__device__ __forceinline__ float lane_seq_sum(float acc, float v, uint32_t lim) {
#pragma unroll
  for (uint32_t t = 0; t < 32; ++t) {
    const float x = __shfl_sync(FULL, v, t);
    if (t < lim) acc += x;
  }
  return acc;
}
__device__ __forceinline__ double lane_seq_sum(double acc, double v, uint32_t lim) {
#pragma unroll
  for (uint32_t t = 0; t < 32; ++t) {
    const double x = __shfl_sync(FULL, v, t);
    if (t < lim) acc += x;
  }
  return acc;
}

// In-order merge of one 32-candidate chunk into a per-ball item list (the slot-map merge of
// pbf.rs:1570-1577 and 2213-2228): candidates with acc = true, taken in lane order, either open a
// new item (appended in first-seen order, initialised with their values) or add their values to
// the existing item of the same fluid index j. slot[] maps j to its item index (NONE when absent)
// and is private to the calling warp. Values: v0 (scalar), v1 (Vec2), v2 (scalar).
struct MergeList {
  uint32_t* j;
  float* v0;
  float2* v1;
  float* v2;  // may be null
  uint32_t cap;
};
__device__ __forceinline__ void warp_merge(bool acc, uint32_t j, float v0, V2 v1, float v2, uint32_t* slot,
                                           const MergeList& L, uint32_t& cnt, bool& overflow) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t key = acc ? j : (0x80000000u | lane);
  const uint32_t peers = __match_any_sync(FULL, key);
  const uint32_t leader = __ffs(peers) - 1;
  uint32_t g = NONE;
  if (acc && lane == leader) g = slot[j];
  const bool is_new = acc && lane == leader && g == NONE;
  const uint32_t newmask = __ballot_sync(FULL, is_new);
  if (is_new) {
    g = cnt + __popc(newmask & ((1u << lane) - 1u));
    if (g < L.cap) { slot[j] = g; L.j[g] = j; } else { overflow = true; }
  }
  cnt += __popc(newmask);
  // the leader of each j (its lowest lane) takes its own value (a new item) or adds it to the
  // stored one, then adds its peers' values in lane order; the rounds run over the largest peer
  // group of the chunk, each round one shuffle per value for all leaders at once
  float a0 = 0.0f, a2 = 0.0f;
  V2 a1;
  const bool lead = acc && lane == leader;
  if (lead) {
    if (is_new) {
      a0 = v0;
      a1 = v1;
      a2 = v2;
    } else if (g < L.cap) {
      a0 = L.v0[g] + v0;
      const V2 s1(L.v1[g]);
      a1 = V2(s1.x + v1.x, s1.y + v1.y);
      a2 = (L.v2 ? L.v2[g] : 0.0f) + v2;
    }
  }
  uint32_t rest = lead ? (peers & (peers - 1u)) : 0u;
  const uint32_t rounds = __reduce_max_sync(FULL, (uint32_t)__popc(rest));
  for (uint32_t k = 0; k < rounds; ++k) {
    const int t = rest ? __ffs(rest) - 1 : (int)lane;
    const float t0 = __shfl_sync(FULL, v0, t), t1x = __shfl_sync(FULL, v1.x, t), t1y = __shfl_sync(FULL, v1.y, t);
    const float t2 = __shfl_sync(FULL, v2, t);
    if (rest) {
      a0 += t0;
      a1.x += t1x;
      a1.y += t1y;
      a2 += t2;
      rest &= rest - 1u;
    }
  }
  if (acc && lane == leader && g < L.cap) {
    L.v0[g] = a0;
    L.v1[g] = a1.f2();
    if (L.v2) L.v2[g] = a2;
  }
  __syncwarp();
}

// Exponent of the value of the lowest set bit of a finite nonzero double: t is an integer
// multiple of 2^granularity_exp(t).
__device__ __forceinline__ int granularity_exp(double t) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(t);
  const int ex = (int)((bits >> 52) & 0x7ffull);
  const unsigned long long mant = bits & 0xfffffffffffffull;
  const unsigned long long sig = ex ? (mant | (1ull << 52)) : mant;
  const int e = ex ? ex - 1075 : -1074;
  return e + __ffsll((long long)sig) - 1;
}

// The f64 sum init + f(0) + ... + f(n-1) when it can be formed in any order with the same bits:
// if every term (and init) is an integer multiple of 2^G and the sum of magnitudes stays below
// 2^(G+52), every partial sum of every order is an integer multiple of 2^G below 2^(G+53) in
// magnitude, exactly representable, so no addition rounds and the left-to-right result equals
// the per-lane-then-tree result computed here. Terms widened from f32 (kinetic energies, wall
// impulses) nearly always qualify. Returns false (and no sum) when the condition fails or a term
// is not finite; the caller then folds in order.
template <class F>
__device__ __forceinline__ bool warp_exact_sum_f64(double init, uint32_t n, F f, double& out) {
  const uint32_t lane = threadIdx.x & 31u;
  double s = 0.0, sabs = 0.0;
  int g = 2000;
  bool finite = true;
  for (uint32_t i = lane; i < n; i += 32) {
    double t = 0.0;
    if (!f(i, t) || t == 0.0) continue;
    if (!isfinite(t)) { finite = false; continue; }
    s += t;
    sabs += fabs(t);
    g = min(g, granularity_exp(t));
  }
  if (lane == 0 && init != 0.0) {
    if (!isfinite(init)) finite = false;
    else {
      s += init;
      sabs += fabs(init);
      g = min(g, granularity_exp(init));
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(FULL, s, o);
    sabs += __shfl_xor_sync(FULL, sabs, o);
    g = min(g, __shfl_xor_sync(FULL, g, o));
  }
  if (!__all_sync(FULL, finite)) return false;
  if (g == 2000) {  // nothing but zero terms: init stays, unless it is a zero itself (sign)
    if (init == 0.0) return false;
    out = init;
    return true;
  }
  if (!(sabs < ldexp(1.0, g + 52))) return false;
  if (s == 0.0) return false;  // an exact zero: its sign depends on the order, fold in order
  out = s;
  return true;
}

// Sequential-order reduction acc = (((init + f(0)) + f(1)) + ...) + f(n-1), with the exact
// rounding of a one-thread loop, computed by one warp: the lanes evaluate 32 consecutive terms in
// parallel (coalesced loads), then every lane adds them in index order by shuffles. Terms for
// which f returns false are skipped (not added). Returns the result to all lanes of the warp.
// f64 sums first try warp_exact_sum_f64, whose result is the same bits when it applies.
template <class T, class F>
__device__ __forceinline__ T warp_ordered_sum(T init, uint32_t n, F f) {
  const uint32_t lane = threadIdx.x & 31u;
  if constexpr (sizeof(T) == 8) {
    double r;
    if (warp_exact_sum_f64(init, n, f, r)) return r;
  }
  T acc = init;
  // software pipeline: the next chunk's terms are evaluated (loads in flight) before the current
  // chunk is folded
  T v = T(0);
  bool use = lane < n ? f(lane, v) : false;
  for (uint32_t c = 0; c < n; c += 32) {
    T vn = T(0);
    bool usen = c + 32 + lane < n ? f(c + 32 + lane, vn) : false;
    const uint32_t mask = __ballot_sync(FULL, use);
    // the 32 shuffles are independent of one another; only the additions form a chain, in lane
    // order, skipping the unused lanes
#pragma unroll
    for (int t = 0; t < 32; ++t) {
      const T x = __shfl_sync(FULL, v, t);
      if ((mask >> t) & 1u) acc += x;
    }
    v = vn;
    use = usen;
  }
  return acc;
}

}  // namespace mg
