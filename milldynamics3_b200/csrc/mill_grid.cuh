// Device uniform grid (grid.rs:101-399 semantics): floor(p / cell) keys, a dense counting-sort CSR
// (cell-key histogram, block prefix scan, scatter, per-cell index sort) when the bounding box
// holds at most 2n + 512 cells, otherwise a sparse layout of sorted occupied keys. Both give the
// reference's iteration order: cells ascending by (cx, cy), points ascending by index in a cell.
#pragma once

#include "mill_block.cuh"

namespace mg {

// Cells with more points than this are filled in index order by a warp instead of sorted (up to
// BIG_LIST such cells per build; further ones are sorted like the rest).
constexpr uint32_t GRID_SMALL_CELL = 32;
constexpr uint32_t BIG_LIST = 64;
constexpr uint32_t BIG_CELL = 0xFFFFFFFFu;  // cursor mark of a cell filled by a warp

__device__ __forceinline__ int2 cell_key(V2 p, float cell) {
  return make_int2(f2i_sat(floorf(p.x / cell)), f2i_sat(floorf(p.y / cell)));
}
__device__ __forceinline__ bool key_lt(int2 a, int2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); }
__device__ __forceinline__ bool key_eq(int2 a, int2 b) { return a.x == b.x && a.y == b.y; }

// Builds the grid of points[0..n) into gb; hdr (shared memory) receives the layout.
// Sets ERR_CELLS in *err if a key saturates the i32 range (coordinates beyond 2^31 cells).
__device__ inline void grid_build(const float2* pts, uint32_t n, float cell, const GridBuf& gb, GridHdr& hdr, uint32_t* err) {
  int32_t mnx = INT32_MAX, mxx = INT32_MIN, mny = INT32_MAX, mxy = INT32_MIN;
  uint32_t cnt = 0;
  bool sat = false;
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 p(pts[i]);
    if (!p.finite()) continue;
    int2 k = cell_key(p, cell);
    gb.pkey[i] = k;
    mnx = min(mnx, k.x); mxx = max(mxx, k.x); mny = min(mny, k.y); mxy = max(mxy, k.y);
    cnt += 1;
    sat = sat || k.x <= INT32_MIN + 1 || k.x >= INT32_MAX - 1 || k.y <= INT32_MIN + 1 || k.y >= INT32_MAX - 1;
  }
  if (sat) atomicOr(err, ERR_CELLS);
  block_minmax_i(mnx, mxx, mny, mxy);
  uint32_t nvalid = block_sum_u(cnt);
  if (tid() == 0) {
    hdr.cell = cell;
    hdr.npoints = nvalid;
    hdr.min_cx = mnx;
    hdr.min_cy = mny;
    hdr.dense = 0;
    hdr.width = hdr.height = 0;
    hdr.ncells = 0;
    if (nvalid > 0) {
      int64_t w = (int64_t)mxx - (int64_t)mnx + 1, h = (int64_t)mxy - (int64_t)mny + 1;
      uint64_t total = (uint64_t)w * (uint64_t)h;
      uint64_t budget = 2ull * nvalid + 512ull;
      if (total <= budget) {
        hdr.dense = 1;
        hdr.width = (int32_t)w;
        hdr.height = (int32_t)h;
        hdr.ncells = (uint32_t)total;
      }
    }
    if (hdr.ncells > gb.cap_cells) { atomicOr(err, ERR_CELLS); hdr.ncells = 0; hdr.dense = 1; hdr.npoints = 0; }
  }
  __syncthreads();
  if (hdr.npoints == 0) {
    if (tid() == 0) { gb.cell_start[0] = 0; hdr.ncells = 0; hdr.dense = 0; }
    __syncthreads();
    return;
  }
  if (hdr.dense) {
    uint32_t total = hdr.ncells;
    for (uint32_t k = tid(); k <= total; k += nthr()) gb.cell_start[k] = 0;
    __syncthreads();
    for (uint32_t i = tid(); i < n; i += nthr()) {
      if (!V2(pts[i]).finite()) continue;
      int2 k = gb.pkey[i];
      uint32_t c = (uint32_t)((k.x - hdr.min_cx) * hdr.height + (k.y - hdr.min_cy));
      atomicAdd(&gb.cell_start[c], 1u);
    }
    __syncthreads();
    block_exclusive_scan(gb.cell_start, total + 1);
    // cells of more than GRID_SMALL_CELL points (up to BIG_LIST of them) are filled in index order
    // by one warp each; the others are scattered by atomics, then sorted by one thread
    __shared__ uint32_t big[BIG_LIST];
    __shared__ uint32_t nbig;
    if (tid() == 0) nbig = 0;
    __syncthreads();
    for (uint32_t k = tid(); k < total; k += nthr()) {
      uint32_t cur = gb.cell_start[k];
      if (gb.cell_start[k + 1] - cur > GRID_SMALL_CELL) {
        const uint32_t q = atomicAdd(&nbig, 1u);
        if (q < BIG_LIST) { big[q] = k; cur = BIG_CELL; }
      }
      gb.cursor[k] = cur;
    }
    __syncthreads();
    for (uint32_t i = tid(); i < n; i += nthr()) {
      if (!V2(pts[i]).finite()) continue;
      int2 k = gb.pkey[i];
      uint32_t c = (uint32_t)((k.x - hdr.min_cx) * hdr.height + (k.y - hdr.min_cy));
      if (gb.cursor[c] == BIG_CELL) continue;
      uint32_t slot = atomicAdd(&gb.cursor[c], 1u);
      gb.indices[slot] = i;
    }
    {
      const uint32_t lane = tid() & 31u, nl = min(nbig, BIG_LIST);
      for (uint32_t q = tid() >> 5; q < nl; q += nthr() >> 5) {
        const uint32_t c = big[q];
        uint32_t o = gb.cell_start[c];
        for (uint32_t c0 = 0; c0 < n; c0 += 32) {
          const uint32_t i = c0 + lane;
          bool hit = false;
          if (i < n && V2(pts[i]).finite()) {
            const int2 k = gb.pkey[i];
            hit = (uint32_t)((k.x - hdr.min_cx) * hdr.height + (k.y - hdr.min_cy)) == c;
          }
          const uint32_t bal = __ballot_sync(0xffffffffu, hit);
          if (hit) gb.indices[o + __popc(bal & ((1u << lane) - 1u))] = i;
          o += __popc(bal);
        }
      }
    }
    __syncthreads();
    for (uint32_t k = tid(); k < total; k += nthr())
      if (gb.cursor[k] != BIG_CELL) small_sort_u32(gb.indices + gb.cell_start[k], gb.cell_start[k + 1] - gb.cell_start[k]);
    __syncthreads();
  } else {
    // Sparse: rank every valid point by (key, index); O(n^2 / threads), used only for a
    // pathologically large bounding box (a diverged point far from the rest).
    for (uint32_t i = tid(); i < n; i += nthr()) {
      if (!V2(pts[i]).finite()) continue;
      int2 ki = gb.pkey[i];
      uint32_t rank = 0;
      for (uint32_t j = 0; j < n; ++j) {
        if (j == i || !V2(pts[j]).finite()) continue;
        int2 kj = gb.pkey[j];
        if (key_lt(kj, ki) || (key_eq(kj, ki) && j < i)) rank += 1;
      }
      gb.indices[rank] = i;
    }
    __syncthreads();
    uint32_t nv = hdr.npoints;
    for (uint32_t q = tid(); q < nv; q += nthr()) {
      bool start = q == 0 || !key_eq(gb.pkey[gb.indices[q]], gb.pkey[gb.indices[q - 1]]);
      gb.cursor[q] = start ? 1u : 0u;
    }
    __syncthreads();
    uint32_t ncell = block_exclusive_scan(gb.cursor, nv);
    for (uint32_t q = tid(); q < nv; q += nthr()) {
      bool start = q == 0 || !key_eq(gb.pkey[gb.indices[q]], gb.pkey[gb.indices[q - 1]]);
      if (start) {
        uint32_t c = gb.cursor[q];
        gb.keys[c] = gb.pkey[gb.indices[q]];
        gb.cell_start[c] = q;
      }
    }
    if (tid() == 0) { gb.cell_start[ncell] = nv; hdr.ncells = ncell; }
    __syncthreads();
  }
}

// grid.rs:242-270 cell_range
__device__ __forceinline__ bool cell_range(const GridHdr& hdr, const GridBuf& gb, int2 key, uint32_t& s, uint32_t& e) {
  if (hdr.npoints == 0) return false;
  if (hdr.dense) {
    int64_t dcx = (int64_t)key.x - hdr.min_cx, dcy = (int64_t)key.y - hdr.min_cy;
    if (dcx < 0 || dcy < 0 || dcx >= hdr.width || dcy >= hdr.height) return false;
    uint32_t k = (uint32_t)(dcx * hdr.height + dcy);
    s = gb.cell_start[k];
    e = gb.cell_start[k + 1];
    return s != e;
  }
  uint32_t lo = 0, hi = hdr.ncells;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (key_lt(gb.keys[mid], key)) lo = mid + 1;
    else hi = mid;
  }
  if (lo >= hdr.ncells || !key_eq(gb.keys[lo], key)) return false;
  s = gb.cell_start[lo];
  e = gb.cell_start[lo + 1];
  return true;
}

// grid.rs:371-399 for_each_near: up to 9 distinct cells, dy outer (-1..1), dx inner (-1..1).
template <class F>
__device__ __forceinline__ void for_each_near(const GridHdr& hdr, const GridBuf& gb, V2 p, F f) {
  if (!p.finite() || hdr.npoints == 0) return;
  int2 c = cell_key(p, hdr.cell);
  int2 ks[9];
  int nk = 0;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      int2 k = make_int2(sat_add(c.x, dx), sat_add(c.y, dy));
      bool seen = false;
      for (int q = 0; q < nk; ++q) seen = seen || key_eq(ks[q], k);
      if (!seen) ks[nk++] = k;
    }
  for (int q = 0; q < nk; ++q) {
    uint32_t s, e;
    if (!cell_range(hdr, gb, ks[q], s, e)) continue;
    for (uint32_t a = s; a < e; ++a) f(gb.indices[a]);
  }
}

// Warp-cooperative for_each_near: the candidates of query point p, in for_each_near order, handed
// out 32 at a time. f(j, pos, valid) is called by every lane of the warp for each chunk, with
// lane l holding candidate pos = chunk start + l (valid = pos < total); f may use warp collectives.
template <class F>
__device__ __forceinline__ void warp_near_chunks(const GridHdr& hdr, const GridBuf& gb, V2 p, F f) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t s = 0, cnt = 0;
  if (p.finite() && hdr.npoints > 0 && lane < 9) {
    int2 c = cell_key(p, hdr.cell);
    int dy = (int)(lane / 3) - 1, dx = (int)(lane % 3) - 1;
    int2 k = make_int2(sat_add(c.x, dx), sat_add(c.y, dy));
    bool dup = false;
    for (uint32_t q = 0; q < lane; ++q) {
      int qy = (int)(q / 3) - 1, qx = (int)(q % 3) - 1;
      dup = dup || key_eq(k, make_int2(sat_add(c.x, qx), sat_add(c.y, qy)));
    }
    uint32_t e;
    if (!dup && cell_range(hdr, gb, k, s, e)) cnt = e - s;
  }
  // inclusive prefix of the 9 cell sizes
  uint32_t incl = cnt;
  for (int o = 1; o < 16; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if ((int)lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 8);
  for (uint32_t c0 = 0; c0 < total; c0 += 32) {
    const uint32_t pos = c0 + lane;
    uint32_t j = NONE;
    // cell of position pos: the first cell whose inclusive prefix exceeds pos
    uint32_t cell = 0, base_prefix = 0, cell_s = 0;
    for (uint32_t q = 0; q < 9; ++q) {
      uint32_t inc_q = __shfl_sync(0xffffffffu, incl, q);
      uint32_t cnt_q = __shfl_sync(0xffffffffu, cnt, q);
      uint32_t s_q = __shfl_sync(0xffffffffu, s, q);
      if (pos < inc_q && pos >= inc_q - cnt_q) { cell = q; base_prefix = inc_q - cnt_q; cell_s = s_q; }
    }
    (void)cell;
    if (pos < total) j = gb.indices[cell_s + (pos - base_prefix)];
    f(j, pos, pos < total);
  }
}

// for_each_near over several query points in turn (point 0's candidates, then point 1's, ...), as
// the per-ball boundary-point loops of pbf.rs:1540-1577 and 2166-2228 visit them, three points
// (27 cell ranges, one per lane) at a time. Lane l of a chunk holds candidate pos = chunk start + l,
// located by a shuffle binary search over the ranges' inclusive prefix. fetch(j, valid) loads
// what f needs of candidate j; it runs one chunk ahead of f, so the next chunk's loads are in
// flight while f works. f(j, q, data, valid) gets the point index q; f may use warp collectives.
template <class PointOf, class Fetch, class F>
__device__ __forceinline__ void warp_near_multi(const GridHdr& hdr, const GridBuf& gb, uint32_t npts, PointOf point_of,
                                                Fetch fetch, F f) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t q0 = 0; q0 < npts; q0 += 3) {
    const uint32_t nq = min(3u, npts - q0);
    uint32_t s = 0, cnt = 0;
    if (lane < 9u * nq && hdr.npoints > 0) {
      const uint32_t c9 = lane % 9u;
      const V2 p = point_of(q0 + lane / 9u);
      if (p.finite()) {
        const int2 c = cell_key(p, hdr.cell);
        const int2 k = make_int2(sat_add(c.x, (int)(c9 % 3u) - 1), sat_add(c.y, (int)(c9 / 3u) - 1));
        bool dup = false;
        for (uint32_t u = 0; u < c9; ++u)
          dup = dup || key_eq(k, make_int2(sat_add(c.x, (int)(u % 3u) - 1), sat_add(c.y, (int)(u / 3u) - 1)));
        uint32_t e;
        if (!dup && cell_range(hdr, gb, k, s, e)) cnt = e - s;
      }
    }
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if ((int)lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    // range r of position pos: the number of ranges whose inclusive prefix is <= pos
    auto locate = [&](uint32_t pos, uint32_t& j, uint32_t& q) {
      uint32_t r = 0;
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t v = __shfl_sync(0xffffffffu, incl, (int)(r + step - 1u));
        if (v <= pos) r += step;
      }
      const uint32_t rs = __shfl_sync(0xffffffffu, s, (int)r), ri = __shfl_sync(0xffffffffu, incl, (int)r);
      const uint32_t rc = __shfl_sync(0xffffffffu, cnt, (int)r);
      q = q0 + r / 9u;
      j = pos < total ? gb.indices[rs + (pos - (ri - rc))] : NONE;
    };
    uint32_t j, q;
    locate(lane, j, q);
    auto d = fetch(j, lane < total);
    for (uint32_t c0 = 0; c0 < total; c0 += 32) {
      const uint32_t nxt = c0 + 32u;
      uint32_t jn = NONE, qn = q0;
      decltype(d) dn{};
      if (nxt < total) {
        locate(nxt + lane, jn, qn);
        dn = fetch(jn, nxt + lane < total);
      }
      f(j, q, d, c0 + lane < total);
      j = jn;
      q = qn;
      d = dn;
    }
  }
}

// The cells a point's neighbour list visits, in the order build_neighbor_lists (pbf.rs:262-288)
// produces: the forward-offset sweep of for_each_candidate_pair (grid.rs:291-362) reaches a point
// in cell C from (-1,-1), (-1,0), (0,-1) before C's own pairs, then C's targets (+1,0), (+1,+1),
// (0,+1), (-1,+1), and finally from (+1,-1). A key at the edge of the i32 range (grid_build sets
// ERR_CELLS then) saturates instead of wrapping, and a stencil cell that saturates onto one already
// visited is not visited again, as in for_each_near.
__constant__ int STENCIL_DX[9] = {-1, -1, 0, 0, 1, 1, 0, -1, 1};
__constant__ int STENCIL_DY[9] = {-1, 0, -1, 0, 0, 1, 1, 1, -1};

template <class F>
__device__ __forceinline__ void for_each_stencil_neighbor(const GridHdr& hdr, const GridBuf& gb, uint32_t self,
                                                          int2 c, F f) {
  // only a key within one cell of the i32 range's ends can saturate
  const bool edge = c.x <= INT32_MIN + 1 || c.x >= INT32_MAX - 1 || c.y <= INT32_MIN + 1 || c.y >= INT32_MAX - 1;
  for (int q = 0; q < 9; ++q) {
    uint32_t s, e;
    const int2 k = make_int2(sat_add(c.x, STENCIL_DX[q]), sat_add(c.y, STENCIL_DY[q]));
    bool dup = false;
    if (edge)
      for (int u = 0; u < q; ++u)
        dup = dup || key_eq(k, make_int2(sat_add(c.x, STENCIL_DX[u]), sat_add(c.y, STENCIL_DY[u])));
    if (dup || !cell_range(hdr, gb, k, s, e)) continue;
    for (uint32_t a = s; a < e; ++a) {
      uint32_t j = gb.indices[a];
      if (j != self) f(j);
    }
  }
}

// Neighbour CSR in the reference's per-particle order (r^2 <= h^2). Two passes: count, scan, fill.
__device__ inline void build_neighbor_lists(const float2* x, uint32_t n, float h, const GridHdr& hdr, const GridBuf& gb,
                                     uint32_t* off, uint32_t* nbrs, uint32_t cap, uint32_t* err, uint32_t* n_edges) {
  float h2 = h * h;
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 xi(x[i]);
    uint32_t c = 0;
    if (xi.finite()) {
      int2 k = cell_key(xi, hdr.cell);
      for_each_stencil_neighbor(hdr, gb, i, k, [&](uint32_t j) {
        if ((xi - V2(x[j])).len2() <= h2) c += 1;
      });
    }
    off[i] = c;
  }
  if (tid() == 0) off[n] = 0;
  __syncthreads();
  uint32_t total = block_exclusive_scan(off, n + 1);
  if (total > cap) {
    if (tid() == 0) atomicOr(err, ERR_EDGES);
    __syncthreads();
    *n_edges = 0;
    return;
  }
  for (uint32_t i = tid(); i < n; i += nthr()) {
    V2 xi(x[i]);
    if (!xi.finite()) continue;
    uint32_t o = off[i];
    int2 k = cell_key(xi, hdr.cell);
    for_each_stencil_neighbor(hdr, gb, i, k, [&](uint32_t j) {
      if ((xi - V2(x[j])).len2() <= h2) nbrs[o++] = j;
    });
  }
  __syncthreads();
  *n_edges = total;
}

// for_each_candidate_pair (grid.rs:291-362) materialised in its visiting order: per occupied cell,
// the in-cell pairs (a < b) then the forward targets (1,0), (1,1), (0,1), (-1,1); each as (min, max).
__constant__ int FWD_DX[4] = {1, 1, 0, -1};
__constant__ int FWD_DY[4] = {0, 1, 1, 1};

__device__ __forceinline__ int2 cell_of(const GridHdr& hdr, const GridBuf& gb, uint32_t k) {
  if (hdr.dense) return make_int2(hdr.min_cx + (int32_t)(k / (uint32_t)hdr.height),
                                  hdr.min_cy + (int32_t)(k % (uint32_t)hdr.height));
  return gb.keys[k];
}

__device__ inline uint32_t build_candidate_pairs(const GridHdr& hdr, const GridBuf& gb, uint32_t* cnt, uint32_t* pi,
                                          uint32_t* pj, uint32_t cap, uint32_t* err) {
  uint32_t nc = hdr.ncells;
  for (uint32_t k = tid(); k < nc; k += nthr()) {
    uint32_t s = gb.cell_start[k], e = gb.cell_start[k + 1];
    uint32_t m = e - s, c = 0;
    if (m > 0) {
      c = m * (m - 1) / 2;
      int2 key = cell_of(hdr, gb, k);
      for (int q = 0; q < 4; ++q) {
        int2 t = make_int2(sat_add(key.x, FWD_DX[q]), sat_add(key.y, FWD_DY[q]));
        if (key_eq(t, key)) continue;
        uint32_t os, oe;
        if (cell_range(hdr, gb, t, os, oe)) c += m * (oe - os);
      }
    }
    cnt[k] = c;
  }
  if (tid() == 0) cnt[nc] = 0;
  __syncthreads();
  uint32_t total = block_exclusive_scan(cnt, nc + 1);
  if (total > cap) {
    if (tid() == 0) atomicOr(err, ERR_PAIRS);
    __syncthreads();
    return 0;
  }
  for (uint32_t k = tid(); k < nc; k += nthr()) {
    uint32_t s = gb.cell_start[k], e = gb.cell_start[k + 1];
    if (s == e) continue;
    uint32_t o = cnt[k];
    for (uint32_t a = s; a < e; ++a)
      for (uint32_t b = a + 1; b < e; ++b) {
        uint32_t i = gb.indices[a], j = gb.indices[b];
        pi[o] = min(i, j); pj[o] = max(i, j); ++o;
      }
    int2 key = cell_of(hdr, gb, k);
    for (int q = 0; q < 4; ++q) {
      int2 t = make_int2(sat_add(key.x, FWD_DX[q]), sat_add(key.y, FWD_DY[q]));
      if (key_eq(t, key)) continue;
      uint32_t os, oe;
      if (!cell_range(hdr, gb, t, os, oe)) continue;
      for (uint32_t a = s; a < e; ++a)
        for (uint32_t b = os; b < oe; ++b) {
          uint32_t i = gb.indices[a], j = gb.indices[b];
          pi[o] = min(i, j); pj[o] = max(i, j); ++o;
        }
    }
  }
  __syncthreads();
  return total;
}

}  // namespace mg
