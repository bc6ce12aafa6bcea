// surface::extract_surface (surface.rs:233-272) on the device, flattened as flatten_polygons
// (surface.rs:420-430) lays it out, in two launches:
//
//  surface_field_kernel    build_field (surface.rs:84-131). One block per 16x16 tile of the
//                          128x128 grid points. Particles stream through shared memory in index
//                          order, compacted to those whose splat box (the reference's rounded
//                          grid-index box) meets the tile, so every grid point adds its terms in
//                          particle order: the same f32 sums as the reference's scatter loop.
//  surface_contour_kernel  polygons_at_threshold (surface.rs:279-351) with the analytic and the
//                          measured-peak thresholds. One block: marching-squares cases and the
//                          per-cell segment prefix live in shared memory; one thread walks the
//                          chains (each grid edge is shared by at most two segments, one in each
//                          adjacent cell, so the candidates of an edge follow from cell arithmetic
//                          in the reference's push order); then all threads interpolate, smooth
//                          and project the points and write the flattened output.
#pragma once

#include "mill_geom.cuh"
#include "mill_kernels.h"

namespace mg {

constexpr float SURF_SPLAT_RADIUS_FACTOR = 1.5f;         // surface.rs:29
constexpr float SURF_THRESHOLD_FRACTION = 0.5f;          // surface.rs:31
constexpr int SURF_TILE = 16;
constexpr int SURF_TILES_AXIS = SURF_G / SURF_TILE;
constexpr uint32_t SURF_NH = SURF_CELLS_AXIS * SURF_G;   // horizontal edges; vertical ones follow
constexpr int SURF_THREADS = 1024;
constexpr uint32_t SURF_CELLS_PER_THREAD = (SURF_CELLS + SURF_THREADS - 1) / SURF_THREADS;
static_assert(SURF_G % SURF_TILE == 0, "tiles cover the grid");
static_assert(SURF_MAX_SEGS < 65536, "segment indices fit 16 bits");

// surface.rs:39-46
__device__ __forceinline__ float surf_splat(float r2, float radius) {
  const float radius2 = radius * radius;
  if (r2 >= radius2) return 0.0f;
  const float t = 1.0f - r2 / radius2;
  return t * t * t;
}
// surface.rs:140-143 (f32::round, clamp, saturating cast: NaN -> 0)
__device__ __forceinline__ uint32_t surf_grid_index(float world, float D, float cell) {
  float raw = roundf((world + D) / cell);
  if (raw < 0.0f) raw = 0.0f;
  if (raw > (float)(SURF_G - 1)) raw = (float)(SURF_G - 1);
  return raw != raw ? 0u : (uint32_t)raw;
}
// surface.rs:145-150
__device__ __forceinline__ V2 surf_grid_point(uint32_t gi, uint32_t gj, float D, float cell) {
  return V2(-D + (float)gi * cell, -D + (float)gj * cell);
}
// glam 0.29 Vec2::lerp: a * (1 - s) + b * s
__device__ __forceinline__ V2 surf_lerp(V2 a, V2 b, float s) {
  return V2(a.x * (1.0f - s) + b.x * s, a.y * (1.0f - s) + b.y * s);
}
// 2.0 * R / (GRID_SIZE as f32 - 1.0)
__device__ __forceinline__ float surf_cell_size(float D) { return 2.0f * D / ((float)SURF_G - 1.0f); }

__global__ void __launch_bounds__(256) surface_field_kernel(const MillDev* __restrict__ mills,
                                                             const StepUniform* __restrict__ uni, SurfDev sd) {
  __shared__ float2 sp[256];
  __shared__ uint32_t sbox[256];
  __shared__ uint32_t wcnt[8];
  const MillDev& m = mills[0];
  const StepUniform& U = *uni;
  const float D = U.drum_radius;
  const uint32_t nf = m.nf;
  const uint32_t tx = blockIdx.x % SURF_TILES_AXIS, ty = blockIdx.x / SURF_TILES_AXIS;
  const uint32_t gi = tx * SURF_TILE + (threadIdx.x % SURF_TILE), gj = ty * SURF_TILE + threadIdx.x / SURF_TILE;
  const float R = SURF_SPLAT_RADIUS_FACTOR * m.f_h;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // surface.rs:71-74
    const float number_density = m.f_rho0 / fmax_r(m.f_mass, 1e-12f);
    *sd.phi_full = number_density * (PI_F * R * R / 4.0f);
  }
  float acc = 0.0f;
  if (nf > 0 && D > 0.0f) {
    const float cell = surf_cell_size(D);
    const V2 gp = surf_grid_point(gi, gj, D, cell);
    const uint32_t ti0 = tx * SURF_TILE, ti1 = ti0 + SURF_TILE - 1;
    const uint32_t tj0 = ty * SURF_TILE, tj1 = tj0 + SURF_TILE - 1;
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (uint32_t base = 0; base < nf; base += 256) {
      const uint32_t i = base + threadIdx.x;
      bool hit = false;
      uint32_t box = 0;
      float2 p = make_float2(0.0f, 0.0f);
      if (i < nf) {
        p = m.fx[i];
        const uint32_t a = surf_grid_index(p.x - R, D, cell), b = surf_grid_index(p.x + R, D, cell);
        const uint32_t c = surf_grid_index(p.y - R, D, cell), d = surf_grid_index(p.y + R, D, cell);
        hit = a <= ti1 && b >= ti0 && c <= tj1 && d >= tj0 && a <= b && c <= d;
        box = a | b << 8 | c << 16 | d << 24;
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, hit);
      if (l == 0) wcnt[w] = __popc(bal);
      __syncthreads();
      uint32_t off = 0, tot = 0;
#pragma unroll
      for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t c = wcnt[k];
        off += k < w ? c : 0u;
        tot += c;
      }
      if (hit) {
        const uint32_t pos = off + __popc(bal & ((1u << l) - 1u));
        sp[pos] = p;
        sbox[pos] = box;
      }
      __syncthreads();
      // Four terms at a time: their divisions overlap, and the sum still takes them in particle
      // order. A particle whose box misses this point adds nothing; adding +0.0 to the running
      // sum (never -0.0: it starts at +0.0 and every term is >= +0.0 or NaN) leaves it unchanged.
      auto term = [&](uint32_t k) {
        const uint32_t bx = sbox[k];
        const float2 q = sp[k];
        const float dx = gp.x - q.x, dy = gp.y - q.y;
        const float v = surf_splat(dx * dx + dy * dy, R);
        const bool in = gi >= (bx & 255u) && gi <= ((bx >> 8) & 255u) && gj >= ((bx >> 16) & 255u) &&
                        gj <= (bx >> 24);
        return in ? v : 0.0f;
      };
      uint32_t k = 0;
      for (; k + 4 <= tot; k += 4) {
        const float t0 = term(k), t1 = term(k + 1), t2 = term(k + 2), t3 = term(k + 3);
        acc += t0;
        acc += t1;
        acc += t2;
        acc += t3;
      }
      for (; k < tot; ++k) acc += term(k);
      __syncthreads();
    }
    // mask with the drum SDF in the drum frame (surface.rs:115-128)
    if (acc != 0.0f && drum_sdf(U, rotate(gp, U.to_local_next)) < 0.0f) acc = 0.0f;
  }
  sd.field[gj * SURF_G + gi] = acc;
}

// Marching-squares segments of each case (surface.rs:194-207): byte 0 the count, bytes 1 and 2
// the pairs of cell sides (0 bottom, 1 right, 2 top, 3 left) as a | b << 4.
#define SURF_PAIR1(a, b) (1u | ((a) | (b) << 4) << 8)
__constant__ uint32_t c_surf_pairs[16] = {
    0u,                   SURF_PAIR1(3u, 0u), SURF_PAIR1(0u, 1u), SURF_PAIR1(3u, 1u),
    SURF_PAIR1(1u, 2u),   2u | (3u | 0u << 4) << 8 | (1u | 2u << 4) << 16,
    SURF_PAIR1(0u, 2u),   SURF_PAIR1(3u, 2u),
    SURF_PAIR1(3u, 2u),   SURF_PAIR1(0u, 2u),
    2u | (0u | 1u << 4) << 8 | (3u | 2u << 4) << 16,
    SURF_PAIR1(1u, 2u),   SURF_PAIR1(3u, 1u), SURF_PAIR1(0u, 1u), SURF_PAIR1(3u, 0u), 0u};
#undef SURF_PAIR1
__device__ __forceinline__ uint32_t surf_case_pairs(uint32_t c) { return c_surf_pairs[c & 15u]; }
// cell_edge_id (surface.rs:209-218) as a dense id: horizontal (i, j) -> j * 127 + i, vertical
// (i, j) -> SURF_NH + j * 128 + i
__device__ __forceinline__ uint32_t surf_edge_id(uint32_t ci, uint32_t cj, uint32_t side) {
  switch (side) {
    case 0: return cj * SURF_CELLS_AXIS + ci;
    case 1: return SURF_NH + cj * SURF_G + ci + 1;
    case 2: return (cj + 1) * SURF_CELLS_AXIS + ci;
    default: return SURF_NH + cj * SURF_G + ci;
  }
}

// Segment links are kept in shared memory up to this many segments, else in global scratch.
constexpr uint32_t SURF_SMALL_SEGS = 4096;
constexpr uint32_t SURF_NONE16 = 0xFFFFu;

struct SurfShared {
  float field[SURF_G * SURF_G];                // the occupancy field
  uint16_t base[SURF_CELLS + 1];               // first segment index of each cell
  uint8_t cases[SURF_CELLS + 3];
  uint32_t visited[(SURF_MAX_SEGS + 31) / 32];
  uint32_t tsum[SURF_THREADS + 1];
  uint32_t seg_e[SURF_SMALL_SEGS];             // edge ids of a segment's ends a | b << 16
  uint32_t seg_n[SURF_SMALL_SEGS];             // segments across a | across b << 16 (SURF_NONE16: none)
};

// Cases of every cell at threshold thr and the exclusive segment prefix; returns the segment
// count. Cell c = cj * 127 + ci; thread t owns cells [t * k, t * k + k).
static __device__ uint32_t surf_cases(SurfShared& sh, float thr) {
  const float* field = sh.field;
  const uint32_t c0 = tid() * SURF_CELLS_PER_THREAD;
  uint32_t cnt = 0;
  for (uint32_t q = 0; q < SURF_CELLS_PER_THREAD; ++q) {
    const uint32_t c = c0 + q;
    if (c >= SURF_CELLS) break;
    const uint32_t ci = c % SURF_CELLS_AXIS, cj = c / SURF_CELLS_AXIS;
    const float* f0 = field + cj * SURF_G + ci;
    const uint32_t cs = (f0[0] > thr ? 1u : 0u) | (f0[1] > thr ? 2u : 0u) | (f0[SURF_G + 1] > thr ? 4u : 0u) |
                        (f0[SURF_G] > thr ? 8u : 0u);
    sh.cases[c] = (uint8_t)cs;
    cnt += surf_case_pairs(cs) & 255u;
  }
  sh.tsum[tid()] = cnt;
  __syncthreads();
  const uint32_t total = block_exclusive_scan(sh.tsum, SURF_THREADS);
  uint32_t run = sh.tsum[tid()];
  for (uint32_t q = 0; q < SURF_CELLS_PER_THREAD; ++q) {
    const uint32_t c = c0 + q;
    if (c >= SURF_CELLS) break;
    sh.base[c] = (uint16_t)run;
    run += surf_case_pairs(sh.cases[c]) & 255u;
  }
  if (tid() == 0) sh.base[SURF_CELLS] = (uint16_t)total;
  __syncthreads();
  return total;
}

// The segment of cell c touching side s, if any: its index and the side of its other end.
__device__ __forceinline__ bool surf_cell_seg(const SurfShared& sh, uint32_t c, uint32_t s, uint32_t& seg,
                                              uint32_t& other) {
  const uint32_t tp = surf_case_pairs(sh.cases[c]);
  const uint32_t n = tp & 255u;
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t pr = (tp >> (8 + 8 * k)) & 255u;
    const uint32_t a = pr & 15u, b = pr >> 4;
    if (a == s || b == s) {
      seg = sh.base[c] + k;
      other = a == s ? b : a;
      return true;
    }
  }
  return false;
}
__device__ __forceinline__ bool surf_visited(const SurfShared& sh, uint32_t s) {
  return (sh.visited[s >> 5] >> (s & 31)) & 1u;
}

// The segment across side `side` of cell (ci, cj): the one touching the same grid edge in the
// neighbouring cell (each crossing edge has exactly one segment end in each cell beside it), or
// SURF_NONE16 at the grid boundary or when the edge does not cross.
__device__ __forceinline__ uint32_t surf_partner(const SurfShared& sh, uint32_t ci, uint32_t cj, uint32_t side) {
  const uint32_t c = cj * SURF_CELLS_AXIS + ci;
  uint32_t nc, opp;
  switch (side) {
    case 0:
      if (cj == 0) return SURF_NONE16;
      nc = c - SURF_CELLS_AXIS; opp = 2; break;
    case 1:
      if (ci + 1 >= (uint32_t)SURF_CELLS_AXIS) return SURF_NONE16;
      nc = c + 1; opp = 3; break;
    case 2:
      if (cj + 1 >= (uint32_t)SURF_CELLS_AXIS) return SURF_NONE16;
      nc = c + SURF_CELLS_AXIS; opp = 0; break;
    default:
      if (ci == 0) return SURF_NONE16;
      nc = c - 1; opp = 1; break;
  }
  uint32_t seg, other;
  return surf_cell_seg(sh, nc, opp, seg, other) ? seg : SURF_NONE16;
}

// Edge ids and partner segments of every segment (all threads): seg_e[s] = a | b << 16 for the
// reference's pair (a, b) of segment s, seg_n[s] = the segments across a and across b. by_edge
// (surface.rs:307-311) lists at most these two segments for an edge, the lower cell's first, so
// extend_chain's "first unvisited candidate" at an edge is the partner of the current segment
// whenever that partner is unvisited.
static __device__ void surf_links(const SurfShared& sh, uint32_t S, uint32_t* seg_e, uint32_t* seg_n) {
  const uint32_t c0 = tid() * SURF_CELLS_PER_THREAD;
  for (uint32_t q = 0; q < SURF_CELLS_PER_THREAD; ++q) {
    const uint32_t c = c0 + q;
    if (c >= SURF_CELLS) break;
    const uint32_t cnt = surf_case_pairs(sh.cases[c]) & 255u;
    for (uint32_t k = 0; k < cnt; ++k) seg_n[sh.base[c] + k] = c | k << 16;
  }
  __syncthreads();
  for (uint32_t sg = tid(); sg < S; sg += nthr()) {
    const uint32_t v = seg_n[sg], c = v & 0xFFFFu, k = v >> 16;
    const uint32_t pr = (surf_case_pairs(sh.cases[c]) >> (8 + 8 * k)) & 255u;
    const uint32_t a = pr & 15u, b = pr >> 4;
    const uint32_t ci = c % SURF_CELLS_AXIS, cj = c / SURF_CELLS_AXIS;
    seg_e[sg] = surf_edge_id(ci, cj, a) | surf_edge_id(ci, cj, b) << 16;
    seg_n[sg] = surf_partner(sh, ci, cj, a) | surf_partner(sh, ci, cj, b) << 16;
  }
  __syncthreads();
}

// extend_chain (surface.rs:371-399), leaving the current segment through edge `in` towards its
// partner `nx`: marks and takes segments until there is no partner or the partner is `stop`,
// appending the far edge of each to dst; returns how many (*closed: it ended at `stop`). In a
// graph where every segment has at most two partners, one per end, a walk from a segment can
// only meet a visited segment again at the segment it started from, so `stop` replaces the
// visited test: the forward walk stops at the start segment of its chain, and the backward walk
// of a chain that did not close meets no visited segment at all.
__device__ __forceinline__ uint32_t surf_extend(SurfShared& sh, const uint32_t* seg_e, const uint32_t* seg_n,
                                                uint32_t in, uint32_t nx, uint32_t stop, uint32_t* dst,
                                                bool* closed) {
  uint32_t n = 0;
  while (nx != SURF_NONE16 && nx != stop) {
    const uint32_t e = seg_e[nx], l = seg_n[nx];
    sh.visited[nx >> 5] |= 1u << (nx & 31);
    const bool in_a = (e & 0xFFFFu) == in;
    const uint32_t ex = in_a ? e >> 16 : e & 0xFFFFu;
    nx = in_a ? l >> 16 : l & 0xFFFFu;
    dst[n++] = ex;
    in = ex;
  }
  *closed = nx == stop && nx != SURF_NONE16;
  return n;
}

// interp_edge (surface.rs:166-187) for a dense edge id
__device__ __forceinline__ V2 surf_interp(const float* __restrict__ field, uint32_t e, float thr, float D,
                                          float cell) {
  uint32_t gi0, gj0, gi1, gj1;
  if (e < SURF_NH) {
    gi0 = e % SURF_CELLS_AXIS; gj0 = e / SURF_CELLS_AXIS; gi1 = gi0 + 1; gj1 = gj0;
  } else {
    const uint32_t v = e - SURF_NH;
    gi0 = v % SURF_G; gj0 = v / SURF_G; gi1 = gi0; gj1 = gj0 + 1;
  }
  const float v0 = field[gj0 * SURF_G + gi0], v1 = field[gj1 * SURF_G + gi1];
  float t;
  if (fabsf(v1 - v0) > 1e-9f) {
    t = (thr - v0) / (v1 - v0);
    if (t < 0.0f) t = 0.0f;
    if (t > 1.0f) t = 1.0f;
  } else {
    t = 0.5f;
  }
  return surf_lerp(surf_grid_point(gi0, gj0, D, cell), surf_grid_point(gi1, gj1, D, cell), t);
}

__global__ void __launch_bounds__(SURF_THREADS) surface_contour_kernel(const MillDev* __restrict__ mills,
                                                                        const StepUniform* __restrict__ uni,
                                                                        SurfDev sd) {
  extern __shared__ __align__(16) unsigned char surf_smem[];
  SurfShared& sh = *reinterpret_cast<SurfShared*>(surf_smem);
  __shared__ float s_thr;
  __shared__ uint32_t s_np, s_npts;
  const MillDev& m = mills[0];
  const StepUniform& U = *uni;
  const float D = U.drum_radius;
  const float* field = sh.field;  // filled below whenever there is a surface
  uint32_t S = 0;
  float thr = 0.0f;
  if (m.nf > 0 && D > 0.0f) {
    const float4* f4 = reinterpret_cast<const float4*>(sd.field);
    float4* s4 = reinterpret_cast<float4*>(sh.field);
    for (uint32_t g = tid(); g < (uint32_t)(SURF_G * SURF_G / 4); g += nthr()) s4[g] = f4[g];
    __syncthreads();
    thr = SURF_THRESHOLD_FRACTION * *sd.phi_full;
    S = surf_cases(sh, thr);
    if (S == 0) {
      // fallback: the grid's measured peak (surface.rs:259-271), fold(0.0, f32::max)
      float pk = 0.0f;
      for (uint32_t g = tid(); g < (uint32_t)(SURF_G * SURF_G); g += nthr()) pk = fmax_r(pk, sh.field[g]);
      for (int o = 16; o > 0; o >>= 1) pk = fmax_r(pk, __shfl_xor_sync(0xffffffffu, pk, o));
      if ((tid() & 31) == 0) sh.tsum[tid() >> 5] = __float_as_uint(pk);
      __syncthreads();
      if (tid() == 0) {
        float p = 0.0f;
        for (uint32_t w = 0; w < nthr() / 32; ++w) p = fmax_r(p, __uint_as_float(sh.tsum[w]));
        s_thr = p;
      }
      __syncthreads();
      const float peak = s_thr;
      __syncthreads();
      if (peak > 0.0f) {
        thr = SURF_THRESHOLD_FRACTION * peak;
        S = surf_cases(sh, thr);
      }
    }
  }
  for (uint32_t k = tid(); k < (S + 31) / 32; k += nthr()) sh.visited[k] = 0u;
  uint32_t* seg_e = S <= SURF_SMALL_SEGS ? sh.seg_e : sd.segs;
  uint32_t* seg_n = S <= SURF_SMALL_SEGS ? sh.seg_n : sd.segs + SURF_MAX_SEGS;
  surf_links(sh, S, seg_e, seg_n);
  if (tid() == 0) {
    // chaining (surface.rs:307-335), one thread
    uint32_t np = 0, woff = 0, npts = 0;
    uint32_t* walk = sd.walk;
    uint32_t* stage = sd.walk + 2 * SURF_MAX_SEGS;
    for (uint32_t start = 0; start < S; ++start) {
      if (surf_visited(sh, start)) continue;
      sh.visited[start >> 5] |= 1u << (start & 31);
      const uint32_t e0 = seg_e[start], l0 = seg_n[start];
      const uint32_t a0 = e0 & 0xFFFFu, b0 = e0 >> 16;
      walk[woff] = a0;
      walk[woff + 1] = b0;
      bool closed = false, unused = false;
      uint32_t n = 2 + surf_extend(sh, seg_e, seg_n, b0, l0 >> 16, start, walk + woff + 2, &closed);
      const uint32_t nbk =
          closed ? 0u : surf_extend(sh, seg_e, seg_n, a0, l0 & 0xFFFFu, SURF_NONE16, stage, &unused);
      if (nbk > 0) {
        // chain = reverse(backward) ++ [a0, b0, forward...]
        for (uint32_t k = n; k-- > 0;) walk[woff + nbk + k] = walk[woff + k];
        for (uint32_t k = 0; k < nbk; ++k) walk[woff + k] = stage[nbk - 1 - k];
        n += nbk;
      }
      if (n > 1 && walk[woff] == walk[woff + n - 1]) --n;
      sd.poly[3 * np] = woff;
      sd.poly[3 * np + 1] = n;
      sd.poly[3 * np + 2] = npts;
      npts += n >= 3 ? 2 * n : n;
      woff += n;
      ++np;
    }
    s_np = np;
    s_npts = npts;
    sd.hdr[0] = 1 + np + 2 * npts;
    sd.hdr[1] = np;
    sd.out[0] = (float)np;
  }
  __syncthreads();
  const uint32_t np = s_np, npts = s_npts;
  if (np == 0) return;
  const float cell = surf_cell_size(D);
  for (uint32_t k = tid(); k < np; k += nthr()) {
    const uint32_t n = sd.poly[3 * k + 1];
    sd.out[1 + k + 2 * sd.poly[3 * k + 2]] = (float)(n >= 3 ? 2 * n : n);
  }
  for (uint32_t q = tid(); q < npts; q += nthr()) {
    // the polygon holding output point q
    uint32_t lo = 0, hi = np - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (sd.poly[3 * mid + 2] <= q) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t off = sd.poly[3 * lo], n = sd.poly[3 * lo + 1], j = q - sd.poly[3 * lo + 2];
    V2 p;
    if (n >= 3) {
      // chaikin_smooth_closed (surface.rs:403-416)
      const uint32_t i = j >> 1, i1 = i + 1 == n ? 0 : i + 1;
      const V2 p0 = surf_interp(field, sd.walk[off + i], thr, D, cell);
      const V2 p1 = surf_interp(field, sd.walk[off + i1], thr, D, cell);
      p = surf_lerp(p0, p1, (j & 1) ? 0.75f : 0.25f);
    } else {
      p = surf_interp(field, sd.walk[off + j], thr, D, cell);
    }
    // project_inside_wall (surface.rs:359-366)
    float d;
    V2 nrm;
    drum_sdf_world(U, p, U.to_local_next, U.to_world_next, d, nrm);
    if (d < 0.0f) p = p - d * nrm;
    float* o = sd.out + 1 + lo + 2 * sd.poly[3 * lo + 2] + 1 + 2 * j;
    o[0] = p.x;
    o[1] = p.y;
  }
}

}  // namespace mg
