// The mill sub-step kernel (one thread block per mill, plus helper blocks for a single mill) and
// its launcher, instantiated per block-size bound in mill_substeps_512.cu and
// mill_substeps_1024.cu (two translation units, so the two instantiations compile in parallel).
#pragma once

#include "mill_dem.cuh"
#include "mill_fluid.cuh"
#include "mill_kernels.h"
#include "mill_stress.cuh"

namespace mg {

// n_sub is the sub-step stride of `angles`; mill b runs n_sub_of[b] sub-steps when n_sub_of is
// given (a batch of mills with different sub-step counts), else n_sub. Two instantiations: up to
// 512 threads per block (128 registers a thread) and up to 1024 (64 registers, more warps for the
// per-ball stages); the results do not depend on the block size. With helpers > 0 the launch runs
// one mill: block 0 is the mill's block and blocks 1..helpers take shares of its per-ball stages
// (mill_wide.cuh); the results do not depend on the number of blocks either. Without helpers,
// block b runs mill block_mill[b] when block_mill is given (an order of the mills, e.g. longest
// first, so that the last wave of blocks holds the short mills), else mill b.
template <int MAX_THREADS>
__global__ void __launch_bounds__(MAX_THREADS) mill_substeps_kernel(const MillDev* __restrict__ mills,
                                                                    StepUniform* uni,
                                                                    const SubAngles* __restrict__ angles,
                                                                    uint32_t n_sub,
                                                                    const uint32_t* __restrict__ n_sub_of,
                                                                    const uint32_t* __restrict__ block_mill,
                                                                    uint32_t helpers) {
  __shared__ MillDev m;
  __shared__ FluidShared fs;
  __shared__ DemShared ds;
  extern __shared__ __align__(16) unsigned char dsm[];  // staged ball state (24 bytes per ball)
  const uint32_t mill = helpers ? 0u : (block_mill ? block_mill[blockIdx.x] : blockIdx.x);
  if (threadIdx.x == 0) {
    m = mills[mill];
    m.helpers = helpers;
    if (blockIdx.x == 0 || helpers == 0) *m.err = 0;
    g_wide_seq = 0;
  }
  __syncthreads();
  if (helpers && blockIdx.x > 0) {
    wide_helper(m, [&](uint32_t phase, const GridHdr& hdr, const float2* vin, float2* vout, uint32_t w0,
                       uint32_t nw) -> uint32_t {
      const StepUniform& U = uni[0];
      const uint32_t t0 = w0 * 32u + (threadIdx.x & 31u), stride = nw * 32u;
      if (phase == WIDE_ADHESION) adhesion_balls(m, U, hdr, w0, nw);
      else if (phase == WIDE_GROUPS) group_balls(m, U, hdr, w0, nw, mill_items(m), w0);
      else if (phase == WIDE_LINKS) return link_balls(m, U, hdr, w0, nw);
      else if (phase == WIDE_DRAG_ITEMS) return drag_item_balls(m, hdr, w0, nw);
      else if (phase == WIDE_BUOYANCY_ITEMS) return buoyancy_item_balls(m, hdr, w0, nw, mill_items(m), m.item_n);
      else if (phase == WIDE_BESIDE_DRAG) return beside_drag(m, U, hdr, fs, dsm);
      else if (phase == WIDE_DRAG_LISTS) return drag_lists(m, U, fs, dsm);
      else if (phase == WIDE_CG_SETUP) cg_setup_rows(m, U.dt, t0, stride);
      else if (phase == WIDE_JOINT_APPLY) joint_apply_rows(m, U.dt, vin, vout, t0, stride);
      else if (phase == WIDE_DRAG_PRE) drag_pre_balls(m, w0, nw);
      else if (phase == WIDE_FLUID_PREP && blockIdx.x == 1) {
        // the next sub-step's fluid steps 0-3, beside the mill block's DEM step
        WideCtl* c = m.wide;
        if (c->tail_out) {
          // the finished sub-step's fluid tail first (it reads the velocities the steps 0-3 change)
          StepOut* to = c->tail_out;
          const unsigned long long tc = fluid_tail(m, c->tail_vmax, c->tail_ke, to->fs, fs);
          if (threadIdx.x == 0) to->stage[12] += tc;
        }
        uint32_t iters = 0;
        unsigned long long cyc[2] = {0, 0};
        fluid_prep(m, U.pbf_iterations, c->prep_dt, fs, &c->prep_err, iters, cyc);
        if (threadIdx.x == 0) {
          c->prep_hdr = fs.hA;
          c->prep_edges = fs.n_edges;
          c->prep_iters = iters;
          c->prep_cycles[0] = cyc[0];
          c->prep_cycles[1] = cyc[1];
        }
      }
      return 0u;
    });
    return;
  }
  const uint32_t my_sub = n_sub_of ? n_sub_of[mill] : n_sub;
  bool prepped = false;  // this sub-step's fluid steps 0-3 were published to helper block 1
  for (uint32_t s = 0; s < my_sub; ++s) {
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
      U.now_s = a.now_s;
      U.alpha = a.alpha;
      memset(&out.ctr, 0, sizeof(out.ctr));
      memset(out.stage, 0, sizeof(out.stage));
      g_stage_last = clock64();
    }
    __syncthreads();
    if (*m.err) break;
    // With helper blocks, the next sub-step's fluid steps 0-3 (they touch only the fluid's arrays,
    // which the DEM step does not) run on helper block 1 while this block runs the DEM step, and
    // so does this sub-step's fluid tail before them; the next fluid step waits for both first.
    const float dt_next = helpers && s + 1 < my_sub ? angles[(size_t)mill * n_sub + s + 1].dt : 0.0f;
    const bool prep_next = helpers && U.run_fluid && s + 1 < my_sub && m.nf > 0 && dt_next > 0.0f;
    // Without the fluid half, imp/ang hold the caller's external impulses (DEM-only entry point).
    double ke_tail = 0.0;
    bool tail_deferred = false;
    if (U.run_fluid) tail_deferred = fluid_step(m, U, out, m.err, fs, dsm, prepped, prep_next, &ke_tail);
    prepped = false;
    __syncthreads();
    if (*m.err) {  // the mill stops; the host reads the error bits from this sub-step's record
      if (threadIdx.x == 0) out.err = *m.err;
      break;
    }
    if (prep_next) {
      const float v_max = fluid_vmax(U);
      wide_publish(m, WIDE_FLUID_PREP, nullptr, nullptr, nullptr, [&](WideCtl* c) {
        c->prep_dt = dt_next;
        c->prep_err = 0u;
        c->tail_out = tail_deferred ? &out : nullptr;
        c->tail_vmax = v_max;
        c->tail_ke = ke_tail;
      });
      prepped = true;
    }
    if (U.run_dem) dem_step(m, U, out, m.impacts + (size_t)s * m.cap_impacts, m.err, ds, dsm);
    __syncthreads();
    if (threadIdx.x == 0) {
      out.stage[14] = out.stage[15] + out.stage[16] + out.stage[17] + out.stage[18] + out.stage[20] + out.stage[21] +
                      out.stage[22] + out.stage[30];
      // Simulation::step's grinding stats: the sub-step's impacts into the stress accumulator
      if (U.fold_stress && !*m.err)
        stress_update(m, m.impacts + (size_t)s * m.cap_impacts, min(out.n_impacts, m.cap_impacts), U.now_s,
                      (double)U.dt, (double)U.alpha, (double)(out.ds.wall_work_j + out.fs.wall_work_j), m.err);
      out.err = *m.err;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && m.stress_copy) *m.stress_copy = *m.stress;
  wide_exit(m);
}

template <int MAX_THREADS>
cudaError_t launch_substeps_impl(const MillDev* mills, uint32_t n_mills, StepUniform* uni, const SubAngles* angles,
                                 uint32_t n_sub, const uint32_t* n_sub_of, uint32_t threads, size_t smem_bytes,
                                 cudaStream_t stream, uint32_t mill_blocks, const uint32_t* block_mill) {
  auto kernel = mill_substeps_kernel<MAX_THREADS>;
  // (the opt-in is needed whenever static plus dynamic shared memory passes 48 KB)
  if (smem_bytes > 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    if (e != cudaSuccess) return e;
  }
  uint32_t helpers = n_mills == 1 && mill_blocks > 1 ? min(mill_blocks, MAX_MILL_BLOCKS) - 1u : 0u;
  if (helpers) {
    // all of the mill's blocks wait for one another, so they must be resident together
    const uint32_t* no_order = nullptr;
    void* args[] = {(void*)&mills,    (void*)&uni,      (void*)&angles, (void*)&n_sub,
                    (void*)&n_sub_of, (void*)&no_order, (void*)&helpers};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)kernel, dim3(1u + helpers), dim3(threads), args,
                                                smem_bytes, stream);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
  }
  kernel<<<n_mills, threads, smem_bytes, stream>>>(mills, uni, angles, n_sub, n_sub_of, block_mill, 0u);
  return cudaGetLastError();
}

}  // namespace mg
