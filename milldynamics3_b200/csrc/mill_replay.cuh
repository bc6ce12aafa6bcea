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
  block_bucket_sort(key, nrec, nbk, start, cur, order, nballs);
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
// balls that share an item. The warps of the block claim balls in index order or by dependency
// level (ball_level_order), and a warp starts ball b once every earlier ball sharing one of b's
// items is done.

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

// Scratch of the dependency levels of a per-ball sweep (32-bit words in shared memory; LEVEL_PREDS
// predecessor slots per ball). A ball's predecessors are the balls that hold the previous record of
// one of its fluid particles; those in the ball's own chunk of 32 balls are kept as a bit mask,
// the others as a set of up to LEVEL_PREDS balls (more: the ball is marked, its records are read
// again when its level is computed).
constexpr uint32_t LEVEL_PREDS = 8;
struct LevelScratch {
  uint32_t* plist;   // LEVEL_PREDS per ball, NONE when free
  uint32_t* over;    // 1: more than LEVEL_PREDS earlier-chunk predecessors
  uint32_t* pmask;   // same-chunk predecessors, bit (p - chunk start)
  uint32_t* lvl;
  uint32_t* order;   // the claim order
  uint32_t* pos;     // position of each ball in the order
  uint32_t* lstart;  // nb + 2 counters (levels are below nb + 1)
};
__device__ inline uint32_t level_scratch_words(uint32_t nb) { return (LEVEL_PREDS + 7u) * nb + 2u; }
__device__ inline bool level_scratch(uint32_t nb, uint32_t* scratch, uint32_t words, LevelScratch& L) {
  if (nb == 0 || scratch == nullptr || words < level_scratch_words(nb)) return false;
  L.plist = scratch;
  L.over = L.plist + LEVEL_PREDS * nb;
  L.pmask = L.over + nb;
  L.lvl = L.pmask + nb;
  L.order = L.lvl + nb;
  L.pos = L.order + nb;
  L.lstart = L.pos + nb;
  return true;
}

// Records ball p as a predecessor of ball b (p < b). Set entries go from NONE to a ball once, so
// concurrent insertions of the same ball leave it once.
__device__ __forceinline__ void level_add_pred(const LevelScratch& L, uint32_t b, uint32_t p) {
  const uint32_t chunk = b & ~31u;
  if (p >= chunk) {
    atomicOr(&L.pmask[b], 1u << (p - chunk));
    return;
  }
  uint32_t* S = L.plist + b * LEVEL_PREDS;
  for (uint32_t i = 0; i < LEVEL_PREDS; ++i) {
    const uint32_t v = atomicCAS(&S[i], NONE, p);
    if (v == NONE || v == p) return;
  }
  L.over[b] = 1u;
}

// rec_pred[r] = the ball of the previous record with the same fluid index (NONE if first). With L,
// also the predecessor sets of the balls (for ball_level_order).
static __device__ void ball_item_preds(const uint32_t* rec_key, const uint32_t* rec_ball, uint32_t nrec, uint32_t nf,
                                       uint32_t nb, uint32_t* start, uint32_t* cur, uint32_t* order, uint32_t* rec_pred,
                                       const LevelScratch* L = nullptr) {
  if (L) {
    for (uint32_t k = tid(); k < LEVEL_PREDS * nb; k += nthr()) L->plist[k] = NONE;
    for (uint32_t b = tid(); b < nb; b += nthr()) { L->over[b] = 0u; L->pmask[b] = 0u; }
  }
  block_bucket_sort(rec_key, nrec, nf, start, cur, order);  // (its barriers order the resets above)
  for (uint32_t j = tid(); j < nf; j += nthr()) {
    uint32_t prev = NONE;
    for (uint32_t q = start[j]; q < start[j + 1]; ++q) {
      const uint32_t r = order[q], b = rec_ball[r];
      rec_pred[r] = prev;
      if (L && prev != NONE) level_add_pred(*L, b, prev);
      prev = b;
    }
  }
  __syncthreads();
}

// A claim order for a per-ball sweep from the predecessor sets ball_item_preds left in L: the balls
// by dependency level (level 0: no predecessor; otherwise one more than the deepest predecessor's
// level), so that the warps of the sweep take the chain's early links first. Every predecessor of
// a ball has a lower level and comes earlier, so claims in this order never wait on a ball that is
// not claimed yet (the order is topological), and the sweep's results do not depend on it.
//   levels (warp 0, chunk after chunk of 32 balls): from the earlier chunks' levels, then the
//          chunk's own dependencies in ball order (lane t's level is final when step t reads it);
//   order: a counting sort by level; pos[] its inverse.
static __device__ const uint32_t* ball_level_order(uint32_t nb, const uint32_t* rec_off, const uint32_t* rec_pred,
                                                   const LevelScratch& L) {
  __shared__ uint32_t s_nlev;
  if (threadIdx.x < 32) {
    const uint32_t lane = threadIdx.x;
    uint32_t maxl = 0;
    for (uint32_t c = 0; c < nb; c += 32) {
      const uint32_t k = c + lane;
      uint32_t base = 0, mk = 0;
      if (k < nb) {
        if (!L.over[k]) {
          const uint32_t* S = L.plist + k * LEVEL_PREDS;
          for (uint32_t i = 0; i < LEVEL_PREDS && S[i] != NONE; ++i) base = max(base, L.lvl[S[i]] + 1u);
        } else {
          for (uint32_t r = rec_off[k]; r < rec_off[k + 1]; ++r) {
            const uint32_t p = rec_pred[r];
            if (p != NONE && p < c) base = max(base, L.lvl[p] + 1u);
          }
        }
        mk = L.pmask[k];
      }
      uint32_t lv = base;
      const uint32_t steps = 32u - __clz(__reduce_or_sync(FULL, mk));  // the highest source lane + 1
      for (uint32_t t = 0; t < steps; ++t) {
        const uint32_t lt = __shfl_sync(FULL, lv, t);
        if ((mk >> t) & 1u) lv = max(lv, lt + 1u);
      }
      if (k < nb) {
        L.lvl[k] = lv;
        maxl = max(maxl, lv + 1u);
      }
      __syncwarp();
    }
    maxl = __reduce_max_sync(FULL, maxl);
    if (lane == 0) s_nlev = maxl;
  }
  __syncthreads();
  const uint32_t nlev = s_nlev;
  for (uint32_t l = tid(); l <= nlev; l += nthr()) L.lstart[l] = 0u;
  __syncthreads();
  for (uint32_t b = tid(); b < nb; b += nthr()) atomicAdd(&L.lstart[L.lvl[b]], 1u);
  __syncthreads();
  block_exclusive_scan(L.lstart, nlev + 1);
  for (uint32_t b = tid(); b < nb; b += nthr()) {
    const uint32_t q = atomicAdd(&L.lstart[L.lvl[b]], 1u);
    L.order[q] = b;
    L.pos[b] = q;
  }
  __syncthreads();
  return L.order;
}

// Whether `order` (positions pos[]) is topological for the records rec_ball / rec_pred: every
// record's predecessor ball comes before the record's ball.
static __device__ bool order_respects(const uint32_t* pos, const uint32_t* rec_ball, const uint32_t* rec_pred,
                                      uint32_t nrec) {
  bool bad = false;
  for (uint32_t r = tid(); r < nrec; r += nthr()) {
    const uint32_t p = rec_pred[r];
    if (p != NONE && !(pos[p] < pos[rec_ball[r]])) bad = true;
  }
  return !__syncthreads_or(bad);
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
// wait only; NONE otherwise). order: the claim order (a topological order such as
// ball_level_order's), or nullptr for index order.
template <class Pre, class Run, class Post>
__device__ void ball_dataflow(uint32_t nb, const uint32_t* rec_off, const uint32_t* rec_pred, uint32_t* done,
                              const uint32_t* order, uint32_t warps, uint32_t spin_ns, uint32_t spin_limit, uint32_t skip_done, uint32_t* err,
                              unsigned long long* acct, Pre pre, Run run, Post post) {
  for (uint32_t b = tid(); b < nb; b += nthr()) done[b] = 0u;
  if (tid() == 0) g_ticket = 0;
  __syncthreads();
  volatile uint32_t* vdone = done;
  const int lane = threadIdx.x & 31;
  // 32-bit clock differences (a ball's parts take far fewer than 2^32 cycles), summed per warp
  uint32_t t_pre = 0, t_wait = 0, t_run = 0;
  for (;;) {
    if ((threadIdx.x >> 5) >= warps) break;
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(&g_ticket, 1u);
    t = __shfl_sync(FULL, t, 0);
    if (t >= nb) break;
    const uint32_t b = order ? order[t] : t;
    const uint32_t t0 = (uint32_t)clock();
    const uint32_t r0 = rec_off[b], r1 = rec_off[b + 1];
    const uint32_t p0 = r0 + lane < r1 ? rec_pred[r0 + lane] : NONE;
    auto st = pre(b, lane);
    const uint32_t t1 = (uint32_t)clock();
    wait_ball_done(vdone, p0, spin_ns, spin_limit, err);
    for (uint32_t c = r0 + 32; c < r1; c += 32)
      wait_ball_done(vdone, c + lane < r1 ? rec_pred[c + lane] : NONE, spin_ns, spin_limit, err);
    __syncwarp();
    __threadfence_block();
    const uint32_t t2 = (uint32_t)clock();
    run(b, lane, st);
    __threadfence_block();
    __syncwarp();
    if (lane == 0 && b != skip_done) vdone[b] = 1u;
    post(b, lane, st);
    t_pre += t1 - t0;
    t_wait += t2 - t1;
    t_run += (uint32_t)clock() - t2;
  }
  if (acct && lane == 0 && (t_pre | t_wait | t_run)) {
    atomicAdd(&acct[0], (unsigned long long)t_pre);
    atomicAdd(&acct[1], (unsigned long long)t_wait);
    atomicAdd(&acct[2], (unsigned long long)t_run);
  }
  __syncthreads();
}

// Three in-order sums over the lanes' values t = 0..lim-1, added to a, b, c (the same on every
// lane): the lanes store their values to the warp's shared scratch, lanes from lim on store -0.0
// (x + -0.0 == x for every x, so padding changes no sum), and lanes 0, 1 and 2 each add one of
// the three in lane order, four at a time from 16-byte loads, the next four's loads in flight
// during the additions; the sums are then broadcast.
__shared__ __align__(16) float g_seq_buf[MAX_BLOCK_WARPS][3][32];
__device__ __forceinline__ void lane_seq_sum3(float& a, float& b, float& c, float va, float vb, float vc,
                                              uint32_t lim) {
  const uint32_t lane = threadIdx.x & 31u;
  float(*B)[32] = g_seq_buf[threadIdx.x >> 5];
  const bool in = lane < lim;
  B[0][lane] = in ? va : -0.0f;
  B[1][lane] = in ? vb : -0.0f;
  B[2][lane] = in ? vc : -0.0f;
  __syncwarp();
  // lanes 0, 1 and 2 each add one of the three sums (one instruction stream for all three)
  if (lane < 3u) {
    const float4* P4 = reinterpret_cast<const float4*>(B[lane]);
    float acc = lane == 0u ? a : (lane == 1u ? b : c);
    const uint32_t groups = (lim + 3u) >> 2;
    float4 x = P4[0];
#pragma unroll
    for (uint32_t g = 0; g < 8; ++g) {
      if (g >= groups) break;
      float4 xn;
      if (g + 1 < 8) xn = P4[g + 1];
      acc += x.x;
      acc += x.y;
      acc += x.z;
      acc += x.w;
      x = xn;
    }
    if (lane == 0u) a = acc;
    else if (lane == 1u) b = acc;
    else c = acc;
  }
  __syncwarp();
  a = __shfl_sync(FULL, a, 0);
  b = __shfl_sync(FULL, b, 1);
  c = __shfl_sync(FULL, c, 2);
}

// One in-order sum over the lanes' values t = 0..lim-1 added to a (the same on every lane), like
// lane_seq_sum3.
__device__ __forceinline__ void lane_seq_sum1(float& a, float va, uint32_t lim) {
  const uint32_t lane = threadIdx.x & 31u;
  float* B = g_seq_buf[threadIdx.x >> 5][0];
  B[lane] = lane < lim ? va : -0.0f;
  __syncwarp();
  if (lane == 0) {
    const float4* A4 = reinterpret_cast<const float4*>(B);
    const uint32_t groups = (lim + 3u) >> 2;
    float4 x = A4[0];
#pragma unroll
    for (uint32_t g = 0; g < 8; ++g) {
      if (g >= groups) break;
      float4 xn;
      if (g + 1 < 8) xn = A4[g + 1];
      a += x.x;
      a += x.y;
      a += x.z;
      a += x.w;
      x = xn;
    }
  }
  __syncwarp();
  a = __shfl_sync(FULL, a, 0);
}

// Block-wide in-order f32 sum init + term(0) + term(1) + ... + term(n-1), every term added (the
// reference's sequential f32 accumulations): all threads evaluate a chunk of terms into shared
// memory (the warps' scratch above, free outside the per-ball sweeps), then thread 0 adds them in
// order with the loads running ahead of the additions. All threads call it; all get the result.
// With SKIP_NONFINITE, non-finite terms are left out (not added).
template <bool SKIP_NONFINITE = false, class Term>
__device__ float block_seq_sum_f32(float init, uint32_t n, Term term) {
  constexpr uint32_t CHUNK = MAX_BLOCK_WARPS * 3 * 32;  // a multiple of 4
  float* buf = &g_seq_buf[0][0][0];
  __shared__ float res;
  float acc = init;
  auto add4 = [&](float4 x) {
    if (!SKIP_NONFINITE || finite_f(x.x)) acc += x.x;
    if (!SKIP_NONFINITE || finite_f(x.y)) acc += x.y;
    if (!SKIP_NONFINITE || finite_f(x.z)) acc += x.z;
    if (!SKIP_NONFINITE || finite_f(x.w)) acc += x.w;
  };
  for (uint32_t c0 = 0; c0 < n; c0 += CHUNK) {
    const uint32_t cnt = min(CHUNK, n - c0), groups = (cnt + 3u) >> 2;
    // the chunk padded with -0.0 to whole groups of four (x + -0.0 == x for every x)
    for (uint32_t k = tid(); k < 4u * groups; k += nthr()) buf[k] = k < cnt ? term(c0 + k) : -0.0f;
    __syncthreads();
    if (tid() == 0) {
      // 16-byte loads two groups ahead of the additions, so that only the chain of additions
      // sets the pace
      const float4* B4 = reinterpret_cast<const float4*>(buf);
      const float4 zero = make_float4(-0.0f, -0.0f, -0.0f, -0.0f);
      float4 x0 = groups > 0 ? B4[0] : zero, x1 = groups > 1 ? B4[1] : zero;
      uint32_t g = 0;
      for (; g + 2 <= groups; g += 2) {
        const float4 x2 = g + 2 < groups ? B4[g + 2] : zero, x3 = g + 3 < groups ? B4[g + 3] : zero;
        add4(x0);
        add4(x1);
        x0 = x2;
        x1 = x3;
      }
      if (g < groups) add4(x0);
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
