// Kernels of the B200 mill sub-step. One thread block owns one mill for the whole launch
// ("mill block"): it runs `n_sub` coupled sub-steps back to back with the mill's state resident in
// HBM/L2, so a batch of mills is one launch with gridDim = number of mills and a plain single mill
// is the same launch with one block.
#include "mill_dem.cuh"
#include "mill_fluid.cuh"
#include "mill_kernels.h"

namespace mg {

__global__ void __launch_bounds__(512) mill_substeps_kernel(const MillDev* __restrict__ mills, StepUniform* uni,
                                                            const SubAngles* __restrict__ angles, uint32_t n_sub) {
  __shared__ MillDev m;
  __shared__ FluidShared fs;
  __shared__ DemShared ds;
  extern __shared__ __align__(16) unsigned char dsm[];  // staged ball state (24 bytes per ball)
  const uint32_t mill = blockIdx.x;
  if (threadIdx.x == 0) m = mills[mill];
  __syncthreads();
  for (uint32_t s = 0; s < n_sub; ++s) {
    StepUniform& U = uni[mill];
    StepOut& out = m.out[s];
    if (threadIdx.x == 0) {
      const SubAngles& a = angles[(size_t)mill * n_sub + s];
      U.drum_angle = a.drum_angle;
      U.drum_angle_next = a.drum_angle_next;
      U.dt = a.dt;
      U.to_local_next = a.to_local_next;
      U.to_world_next = a.to_world_next;
      U.to_local0 = a.to_local0;
      memset(&out.ctr, 0, sizeof(out.ctr));
      memset(out.stage, 0, sizeof(out.stage));
      g_stage_last = clock64();
    }
    __syncthreads();
    if (*m.err) break;
    // Without the fluid half, imp/ang hold the caller's external impulses (DEM-only entry point).
    if (U.run_fluid) fluid_step(m, U, out, m.err, fs, dsm);
    __syncthreads();
    if (*m.err) break;
    if (U.run_dem) dem_step(m, U, out, m.impacts + (size_t)s * m.cap_impacts, m.err, ds, dsm);
    __syncthreads();
    if (threadIdx.x == 0) out.stage[14] = out.stage[15] + out.stage[16] + out.stage[17] + out.stage[18] + out.stage[20] + out.stage[21] + out.stage[22] + out.stage[30];
    if (threadIdx.x == 0) out.err = *m.err;
    __syncthreads();
  }
}

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
                            uint32_t n_sub, uint32_t threads, size_t smem_bytes, cudaStream_t stream) {
  if (threads == 0 || threads > 512) threads = 512;
  if (smem_bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(mill_substeps_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bytes);
    if (e != cudaSuccess) return e;
  }
  mill_substeps_kernel<<<n_mills, threads, smem_bytes, stream>>>(mills, uni, angles, n_sub);
  return cudaGetLastError();
}

cudaError_t launch_probe(const MillDev* mill, float cell, int mode, uint32_t* result, cudaStream_t stream) {
  probe_kernel<<<1, 512, 0, stream>>>(mill, cell, mode, result);
  return cudaGetLastError();
}

}  // namespace mg
