// Kernels of the B200 mill sub-step. One thread block owns one mill for the whole launch
// ("mill block"): it runs `n_sub` coupled sub-steps back to back with the mill's state resident in
// HBM/L2, so a batch of mills is one launch with gridDim = number of mills and a plain single mill
// is the same launch with one block. The sub-step kernel itself is in mill_substeps.cuh
// (instantiated in mill_substeps_512.cu / mill_substeps_1024.cu); this file holds its dispatch and
// the grid probe, impact packing, metrics and free-surface kernels.
#include "mill_grid.cuh"
#include "mill_kernels.h"
#include "mill_metrics.cuh"
#include "mill_surface.cuh"

namespace mg {

// Grid-stage probe: builds the grid of caller points and, per `mode`, leaves the grid (0), the
// candidate pairs (1) or the neighbour CSR (2) in the descriptor's buffers.
__global__ void __launch_bounds__(512) probe_kernel(const MillDev* __restrict__ mills, float cell, int mode,
                                                    uint32_t* __restrict__ result) {
  __shared__ MillDev m;
  __shared__ GridHdr hdr;
  __shared__ uint32_t n_edges;
  if (threadIdx.x == 0) m = mills[0];
  __syncthreads();
  grid_build(m.fx, m.nf, cell, m.gA, hdr, m.err);
  if (mode == 1) {
    uint32_t np = build_candidate_pairs(hdr, m.gA, m.pair_cnt, m.pair_i, m.pair_j, m.cap_pairs, m.err);
    if (threadIdx.x == 0) result[8] = np;
  } else if (mode == 2) {
    build_neighbor_lists(m.fx, m.nf, cell, hdr, m.gA, m.nbr_off, m.nbrs, m.cap_edges, m.err, &n_edges);
    if (threadIdx.x == 0) result[8] = n_edges;
  }
  if (threadIdx.x == 0) {
    result[0] = (uint32_t)hdr.dense;
    result[1] = (uint32_t)hdr.min_cx;
    result[2] = (uint32_t)hdr.min_cy;
    result[3] = (uint32_t)hdr.width;
    result[4] = (uint32_t)hdr.height;
    result[5] = hdr.ncells;
    result[6] = hdr.npoints;
    result[7] = *m.err;
  }
}

cudaError_t launch_substeps(const MillDev* mills, uint32_t n_mills, StepUniform* uni, const SubAngles* angles,
                            uint32_t n_sub, const uint32_t* n_sub_of, uint32_t threads, size_t smem_bytes,
                            cudaStream_t stream, uint32_t mill_blocks, const uint32_t* block_mill, bool regs64) {
  if (threads == 0 || threads > MAX_BLOCK_THREADS) threads = DEFAULT_BLOCK_THREADS;
  if (threads > 512 || regs64)
    return launch_substeps_1024(mills, n_mills, uni, angles, n_sub, n_sub_of, threads, smem_bytes, stream,
                                mill_blocks, block_mill);
  return launch_substeps_512(mills, n_mills, uni, angles, n_sub, n_sub_of, threads, smem_bytes, stream, mill_blocks,
                             block_mill);
}

// One block per mill: appends the mill's impact records (sub-step order) to the packed buffer.
__global__ void __launch_bounds__(256) pack_impacts_kernel(const MillDev* __restrict__ mills,
                                                           const uint32_t* __restrict__ n_sub_of,
                                                           MgImpactRecord* packed, uint32_t cap, uint32_t* cursor,
                                                           uint2* table) {
  __shared__ uint32_t base;
  const uint32_t mill = blockIdx.x;
  const MillDev& m = mills[mill];
  const uint32_t ns = n_sub_of[mill];
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t s = 0; s < ns; ++s) t += min(m.out[s].n_impacts, m.cap_impacts);
    base = atomicAdd(cursor, t);
    table[mill] = make_uint2(base, t);
  }
  __syncthreads();
  uint32_t o = base;
  for (uint32_t s = 0; s < ns; ++s) {
    const uint32_t ni = min(m.out[s].n_impacts, m.cap_impacts);
    const MgImpactRecord* src = m.impacts + (size_t)s * m.cap_impacts;
    for (uint32_t r = threadIdx.x; r < ni; r += blockDim.x)
      if (o + r < cap) packed[o + r] = src[r];
    o += ni;
  }
}

cudaError_t launch_pack_impacts(const MillDev* mills, uint32_t n_mills, const uint32_t* n_sub_of,
                                MgImpactRecord* packed, uint32_t cap, uint32_t* cursor, uint2* table,
                                cudaStream_t stream) {
  pack_impacts_kernel<<<n_mills, 256, 0, stream>>>(mills, n_sub_of, packed, cap, cursor, table);
  return cudaGetLastError();
}

cudaError_t launch_metrics(const MillDev* mill, const StepUniform* uni, MgMetrics* out, cudaStream_t stream) {
  metrics_kernel<<<1, 1024, 0, stream>>>(mill, uni, out);
  return cudaGetLastError();
}

cudaError_t launch_surface(const MillDev* mill, const StepUniform* uni, const SurfDev& sd, bool contour,
                           cudaStream_t stream) {
  surface_field_kernel<<<SURF_TILES_AXIS * SURF_TILES_AXIS, SURF_TILE * SURF_TILE, 0, stream>>>(mill, uni, sd);
  if (contour) {
    cudaError_t e = cudaFuncSetAttribute(surface_contour_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(SurfShared));
    if (e != cudaSuccess) return e;
    surface_contour_kernel<<<1, SURF_THREADS, sizeof(SurfShared), stream>>>(mill, uni, sd);
  }
  return cudaGetLastError();
}

cudaError_t launch_probe(const MillDev* mill, float cell, int mode, uint32_t* result, cudaStream_t stream) {
  probe_kernel<<<1, 512, 0, stream>>>(mill, cell, mode, result);
  return cudaGetLastError();
}

}  // namespace mg
