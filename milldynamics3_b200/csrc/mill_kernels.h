// Host-visible launch wrappers of mill_kernels.cu.
#pragma once

#include "mill_common.cuh"

namespace mg {

// Runs coupled sub-steps on each of n_mills mills (one block per mill): n_sub_of[b] of them on
// mill b when n_sub_of is given, else n_sub. uni holds one StepUniform per mill; angles holds
// n_mills * n_sub SubAngles, mill-major (n_sub is the stride). Each mill's sticky error word is
// cleared at the start of the launch. smem_bytes of dynamic shared memory must be at least every
// mill's MillDev::smem_bytes. With n_mills == 1 and mill_blocks > 1, the mill's per-ball stages
// are shared with mill_blocks - 1 helper blocks (a cooperative launch; the mill's control block
// must be zeroed before the launch and its slot maps sized for all the blocks' warps). Without
// helpers, block b runs mill block_mill[b] when block_mill is given. The instantiation: blocks of
// more than 512 threads, or any block size with regs64, run the 64-register build (two 512-thread
// blocks fit one SM); otherwise the 128-register build of up to 512 threads.
cudaError_t launch_substeps(const MillDev* mills, uint32_t n_mills, StepUniform* uni, const SubAngles* angles,
                            uint32_t n_sub, const uint32_t* n_sub_of, uint32_t threads, size_t smem_bytes,
                            cudaStream_t stream, uint32_t mill_blocks = 1, const uint32_t* block_mill = nullptr,
                            bool regs64 = false);
// The two instantiations behind launch_substeps (blocks of up to 512 and up to 1024 threads).
cudaError_t launch_substeps_512(const MillDev* mills, uint32_t n_mills, StepUniform* uni, const SubAngles* angles,
                                uint32_t n_sub, const uint32_t* n_sub_of, uint32_t threads, size_t smem_bytes,
                                cudaStream_t stream, uint32_t mill_blocks, const uint32_t* block_mill);
cudaError_t launch_substeps_1024(const MillDev* mills, uint32_t n_mills, StepUniform* uni, const SubAngles* angles,
                                 uint32_t n_sub, const uint32_t* n_sub_of, uint32_t threads, size_t smem_bytes,
                                 cudaStream_t stream, uint32_t mill_blocks, const uint32_t* block_mill);
// Packs the impact records of n_mills mills after a launch: mill b's records of its sub-steps
// 0..n_sub_of[b]-1 (StepOut::n_impacts each, at most cap_impacts) are appended in sub-step order
// at an offset taken from *cursor (one atomic per mill); table[b] = {offset, count}. Records that
// would pass `cap` are not written (the count still is).
cudaError_t launch_pack_impacts(const MillDev* mills, uint32_t n_mills, const uint32_t* n_sub_of,
                                MgImpactRecord* packed, uint32_t cap, uint32_t* cursor, uint2* table,
                                cudaStream_t stream);
// Largest dynamic shared-memory allotment of a launch. The region holds, one phase at a time,
// the fluid positions and velocities plus completion flags of the drag / buoyancy sweeps
// (16 nf + 4 nb bytes) and the ball state of the DEM sweeps (24 nb bytes), with sweep_scratch
// also the projection sweep's scratch after it (16 bytes per item, reserved for 8 items a ball,
// and 4 nb of excursions); it is sized to the largest of them (without the projection scratch
// when that does not fit), and the rest of the SM's L1 / shared storage stays L1 cache. Batches
// leave the projection scratch out: the L1 it takes costs more across mills than it saves.
constexpr size_t MAX_STAGE_SMEM = 200 * 1024;
inline size_t stage_smem_bytes(uint32_t nf, uint32_t nb, bool sweep_scratch) {
  const size_t fluid = 16 * (size_t)nf + 4 * (size_t)nb + 64, balls = 24 * (size_t)nb;
  const size_t sweep = sweep_scratch ? balls + 16 + 132 * (size_t)nb : balls;
  auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
  const size_t want = up(fluid > sweep ? fluid : sweep);
  if (want <= MAX_STAGE_SMEM) return want;
  const size_t need = up(fluid > balls ? fluid : balls);
  if (need <= MAX_STAGE_SMEM) return need;
  return up(balls) <= MAX_STAGE_SMEM ? up(balls) : 0;
}
// Sets the message mg_global_last_error() returns on this host thread; returns code.
int set_global_error(int code, const char* msg);
// metrics::compute on mill[0]'s state (one block); uni holds the mill's geometry with
// to_local_next / to_world_next set for the current drum angle.
cudaError_t launch_metrics(const MillDev* mill, const StepUniform* uni, MgMetrics* out, cudaStream_t stream);

// Free-surface extraction (surface.rs:233-272): the 128 x 128 grid points over [-R, R] of the
// occupancy field, and its (128 - 1)^2 marching-squares cells with at most two segments each.
constexpr int SURF_G = MG_SURFACE_GRID;
constexpr int SURF_CELLS_AXIS = SURF_G - 1;
constexpr int SURF_CELLS = SURF_CELLS_AXIS * SURF_CELLS_AXIS;
constexpr uint32_t SURF_MAX_SEGS = 2 * SURF_CELLS;
// chains hold at most S + P <= 2 S edge ids (S segments, P polygons), and backward walks stage
// at most S more
constexpr uint32_t SURF_WALK_CAP = 3 * SURF_MAX_SEGS;
// 1 + P + 2 T floats with T <= 2 (S + P) smoothed points
constexpr uint32_t SURF_OUT_CAP = 1 + 9 * SURF_MAX_SEGS;
// Device scratch of the free-surface launches.
struct SurfDev {
  float* field;      // SURF_G^2, row gj * SURF_G + gi
  uint32_t* segs;    // segment edge ids and partners when they exceed shared memory (2 S)
  uint32_t* walk;    // chains (edge ids), then backward-walk staging
  uint32_t* poly;    // per polygon: chain offset, chain length, first output point
  float* out;        // flattened polygons
  uint32_t* hdr;     // [0] output floats, [1] polygons
  float* phi_full;   // analytic_phi_full of the fluid
};
// The occupancy field and phi_full of mill 0 (one launch), then with `contour` the flattened
// polygons into sd.out and their length into sd.hdr[0] (a second launch).
cudaError_t launch_surface(const MillDev* mill, const StepUniform* uni, const SurfDev& sd, bool contour,
                           cudaStream_t stream);
// Grid-stage probe over the descriptor's fx[0..nf): mode 0 grid, 1 candidate pairs, 2 neighbours.
cudaError_t launch_probe(const MillDev* mill, float cell, int mode, uint32_t* result, cudaStream_t stream);

}  // namespace mg
