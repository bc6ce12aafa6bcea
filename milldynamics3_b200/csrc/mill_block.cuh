// Block-level building blocks for the one-CTA-per-mill kernels: deterministic reductions, an
// in-place exclusive scan over global memory, and a stable bucket sort (records grouped by key,
// ascending record index inside a bucket). Every routine is called by all threads of the block.
#pragma once

#include "mill_common.cuh"

namespace mg {

__device__ __forceinline__ uint32_t tid() { return threadIdx.x; }

// Stage timing: thread 0 adds the cycles since the previous mark to out_stage[slot]. Called right
// after a block barrier, so the interval covers the whole block's work on the stage.
__shared__ long long g_stage_last;
__device__ __forceinline__ void stage_mark(unsigned long long* out_stage, int slot) {
  if (threadIdx.x == 0) {
    long long t = clock64();
    out_stage[slot] += (unsigned long long)(t - g_stage_last);
    g_stage_last = t;
  }
}
__device__ __forceinline__ uint32_t nthr() { return blockDim.x; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic f64 sum: fixed xor-tree inside warps, then a fixed tree over the warp sums.
__device__ inline double block_sum_d(double v) {
  __shared__ double sh[32];
  __shared__ double res;
  v = warp_sum(v);
  int w = tid() >> 5, l = tid() & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    int nw = (nthr() + 31) >> 5;
    double x = l < nw ? sh[l] : 0.0;
    x = warp_sum(x);
    if (l == 0) res = x;
  }
  __syncthreads();
  double r = res;
  __syncthreads();
  return r;
}

__device__ inline uint32_t block_sum_u(uint32_t v) {
  __shared__ uint32_t sh[32];
  __shared__ uint32_t res;
  v = warp_sum(v);
  int w = tid() >> 5, l = tid() & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    int nw = (nthr() + 31) >> 5;
    uint32_t x = l < nw ? sh[l] : 0u;
    x = warp_sum(x);
    if (l == 0) res = x;
  }
  __syncthreads();
  uint32_t r = res;
  __syncthreads();
  return r;
}

// f32::max fold (order-independent: max is exact).
__device__ inline float block_max_f(float v) {
  __shared__ float sh[32];
  __shared__ float res;
  for (int o = 16; o > 0; o >>= 1) v = fmax_r(v, __shfl_xor_sync(0xffffffffu, v, o));
  int w = tid() >> 5, l = tid() & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    int nw = (nthr() + 31) >> 5;
    float x = l < nw ? sh[l] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) x = fmax_r(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (l == 0) res = x;
  }
  __syncthreads();
  float r = res;
  __syncthreads();
  return r;
}

__device__ inline void block_minmax_i(int32_t& mn0, int32_t& mx0, int32_t& mn1, int32_t& mx1) {
  __shared__ int32_t sh[4][32];
  int w = tid() >> 5, l = tid() & 31;
  for (int o = 16; o > 0; o >>= 1) {
    mn0 = min(mn0, __shfl_xor_sync(0xffffffffu, mn0, o));
    mx0 = max(mx0, __shfl_xor_sync(0xffffffffu, mx0, o));
    mn1 = min(mn1, __shfl_xor_sync(0xffffffffu, mn1, o));
    mx1 = max(mx1, __shfl_xor_sync(0xffffffffu, mx1, o));
  }
  if (l == 0) { sh[0][w] = mn0; sh[1][w] = mx0; sh[2][w] = mn1; sh[3][w] = mx1; }
  __syncthreads();
  int nw = (nthr() + 31) >> 5;
  mn0 = INT32_MAX; mx0 = INT32_MIN; mn1 = INT32_MAX; mx1 = INT32_MIN;
  for (int k = 0; k < nw; ++k) {
    mn0 = min(mn0, sh[0][k]); mx0 = max(mx0, sh[1][k]);
    mn1 = min(mn1, sh[2][k]); mx1 = max(mx1, sh[3][k]);
  }
  __syncthreads();
}

// In-place exclusive scan of a[0..m); returns the total. All threads call it.
__device__ inline uint32_t block_exclusive_scan(uint32_t* a, uint32_t m) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry;
  if (tid() == 0) carry = 0;
  __syncthreads();
  int w = tid() >> 5, l = tid() & 31;
  int nw = (nthr() + 31) >> 5;
  for (uint32_t base = 0; base < m; base += nthr()) {
    uint32_t idx = base + tid();
    uint32_t v = idx < m ? a[idx] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (l >= o) x += y;
    }
    if (l == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      uint32_t s = l < nw ? wsum[l] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (l >= o) s += y;
      }
      if (l < nw) wsum[l] = s;  // inclusive warp prefix
    }
    __syncthreads();
    uint32_t before = carry + (w > 0 ? wsum[w - 1] : 0u) + (x - v);
    if (idx < m) a[idx] = before;
    __syncthreads();
    if (tid() == 0) carry += wsum[nw - 1];
    __syncthreads();
  }
  uint32_t total = carry;
  __syncthreads();
  return total;
}

// Sorts a[0..n), n <= N, in registers: one batch of loads, a bitonic network (the tail padded
// with the largest value), one batch of stores.
template <int N>
__device__ __forceinline__ void reg_sort_u32(uint32_t* a, uint32_t n) {
  uint32_t v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = (uint32_t)k < n ? a[k] : 0xFFFFFFFFu;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const uint32_t x = v[i], y = v[l];
          if ((x > y) == up) {
            v[i] = y;
            v[l] = x;
          }
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < N; ++k)
    if ((uint32_t)k < n) a[k] = v[k];
}

// Sort of a short segment (ascending): in registers up to 32 entries, else insertion sort.
__device__ __forceinline__ void small_sort_u32(uint32_t* a, uint32_t n) {
  if (n <= 1) return;
  if (n <= 8) { reg_sort_u32<8>(a, n); return; }
  if (n <= 32) { reg_sort_u32<32>(a, n); return; }
  for (uint32_t i = 1; i < n; ++i) {
    uint32_t v = a[i];
    uint32_t j = i;
    while (j > 0 && a[j - 1] > v) { a[j] = a[j - 1]; --j; }
    a[j] = v;
  }
}

// Ascending sort of a[0..n), n <= 256, by one full warp: element e = 32 r + lane sits in lane
// `lane`'s register r (the tail padded with the largest value); a bitonic network whose
// partners are 32 or more apart swap registers and the nearer ones exchange by shuffles.
__device__ __forceinline__ void warp_sort256_u32(uint32_t* a, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t v[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const uint32_t e = 32u * r + lane;
    v[r] = e < n ? a[e] : 0xFFFFFFFFu;
  }
#pragma unroll
  for (uint32_t k = 2; k <= 256; k <<= 1) {
#pragma unroll
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const uint32_t rj = j >> 5;
#pragma unroll
        for (uint32_t r = 0; r < 8; ++r) {
          const uint32_t rr = r ^ rj;
          if (rr > r) {
            const bool up = ((32u * r + lane) & k) == 0;
            const uint32_t x = v[r], y = v[rr];
            if ((x > y) == up) { v[r] = y; v[rr] = x; }
          }
        }
      } else {
#pragma unroll
        for (uint32_t r = 0; r < 8; ++r) {
          const uint32_t y = __shfl_xor_sync(0xffffffffu, v[r], (int)j);
          const bool up = ((32u * r + lane) & k) == 0;
          const bool lower = (lane & j) == 0;
          v[r] = lower == up ? min(v[r], y) : max(v[r], y);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const uint32_t e = 32u * r + lane;
    if (e < n) a[e] = v[r];
  }
}

// Stable bucket sort: start[0..nbk] receives bucket offsets, order[] the record indices grouped by
// key in ascending record order; cur[0..nbk) is scratch. Only the first nsorted buckets (all when
// nsorted >= nbk) are filled: the records of later buckets are counted in start[] but their part of
// order[] is left unwritten (for a bucket that collects records nobody reads).
__device__ inline void block_bucket_sort(const uint32_t* keys, uint32_t nrec, uint32_t nbk, uint32_t* start, uint32_t* cur,
                                  uint32_t* order, uint32_t nsorted = 0xFFFFFFFFu) {
  for (uint32_t k = tid(); k <= nbk; k += nthr()) start[k] = 0;
  __syncthreads();
  for (uint32_t r = tid(); r < nrec; r += nthr()) atomicAdd(&start[keys[r]], 1u);
  __syncthreads();
  block_exclusive_scan(start, nbk + 1);
  // Buckets of up to 32 records: scattered by atomics, then sorted by one thread. 33 to 256
  // records (up to 256 such buckets): scattered, then sorted by one warp in registers. More than
  // 256 (up to 64 such buckets): filled in record order by one warp. Buckets beyond those lists
  // are scattered and sorted by one thread.
  constexpr uint32_t SMALL = 32, MID = 256, NMID = 256, NBIG = 64;
  constexpr uint32_t BIG_MARK = 0xFFFFFFFFu, MID_MARK = 0xFFFFFFFEu;
  __shared__ uint32_t big[NBIG], mid[NMID];
  __shared__ uint32_t nbig, nmid;
  if (tid() == 0) { nbig = 0; nmid = 0; }
  __syncthreads();
  for (uint32_t k = tid(); k < nbk; k += nthr()) {
    uint32_t c = start[k];
    const uint32_t sz = start[k + 1] - c;
    if (k >= nsorted) {
      c = BIG_MARK;  // not filled
    } else if (sz > MID) {
      const uint32_t q = atomicAdd(&nbig, 1u);
      if (q < NBIG) { big[q] = k; c = BIG_MARK; }
    } else if (sz > SMALL) {
      const uint32_t q = atomicAdd(&nmid, 1u);
      if (q < NMID) mid[q] = k;
    }
    cur[k] = c;
  }
  __syncthreads();
  for (uint32_t r = tid(); r < nrec; r += nthr()) {
    const uint32_t k = keys[r];
    if (cur[k] == BIG_MARK) continue;
    uint32_t slot = atomicAdd(&cur[k], 1u);
    order[slot] = r;
  }
  __syncthreads();
  const uint32_t nl_mid = min(nmid, NMID), nl_big = min(nbig, NBIG);
  for (uint32_t q = tid(); q < nl_mid; q += nthr()) cur[mid[q]] = MID_MARK;
  {
    const uint32_t lane = tid() & 31u;
    for (uint32_t q = tid() >> 5; q < nl_mid + nl_big; q += nthr() >> 5) {
      if (q < nl_mid) {
        const uint32_t k = mid[q];
        warp_sort256_u32(order + start[k], start[k + 1] - start[k]);
        continue;
      }
      const uint32_t k = big[q - nl_mid];
      uint32_t o = start[k];
      for (uint32_t c0 = 0; c0 < nrec; c0 += 32) {
        const uint32_t r = c0 + lane;
        const bool hit = r < nrec && keys[r] == k;
        const uint32_t bal = __ballot_sync(0xffffffffu, hit);
        if (hit) order[o + __popc(bal & ((1u << lane) - 1u))] = r;
        o += __popc(bal);
      }
    }
  }
  __syncthreads();
  for (uint32_t k = tid(); k < nbk; k += nthr())
    if (cur[k] < MID_MARK) small_sort_u32(order + start[k], start[k + 1] - start[k]);
  __syncthreads();
}

}  // namespace mg
