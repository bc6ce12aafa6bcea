// Fluid neighbour lists (grid build + CSR, pbf.rs:262-288 over grid.rs:101-285) with no
// allocation at all: the one entry point of the library that never calls cudaMalloc/cudaFree and
// uses no allocating library.
//
// Who needs it. A caller that runs the sub-step inside a fixed device-memory budget (a serving
// loop that admits mills by their measured footprint) or inside a frame loop that must not stall
// (cudaMalloc and cudaFree synchronise the device, which would stall every other mill's stream)
// cannot allocate per call. mg_probe_neighbor_lists allocates a temporary arena on every call;
// this variant takes its grid scratch from one fixed static device array instead and reads and
// writes only caller-owned device memory, asynchronously on the caller's stream.
//
// Limits and rules:
//   * at most NOALLOC_MAX_POINTS points per call (larger requests are rejected with
//     MG_ERR_CAPACITY before anything runs); the scratch is ~0.6 MB per device;
//   * nothing in the scratch has to start at zero: the kernel writes every scratch word before it
//     reads it in the same call, and its error word lives in shared memory;
//   * the scratch is shared by all calls on one device, so calls on the same device must not
//     overlap: issue them on one stream, or order them with events. Overlapping calls race on the
//     scratch and give undefined results;
//   * the first call on a device resolves the scratch's address (cudaGetSymbolAddress) once; make
//     that first call before capturing a stream;
//   * that address is cached per device ordinal for the life of the process and is valid in the
//     device's primary context only (the one the CUDA runtime uses): a cudaDeviceReset between
//     calls, or a call made while another context is current on the device, would hand the kernel
//     a stale address, so neither is allowed.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "mill_grid.cuh"
#include "mill_kernels.h"
#include "../../include/millgpu.h"

namespace mg {

namespace {

constexpr uint32_t NOALLOC_MAX_POINTS = 16384;
constexpr uint32_t NOALLOC_MAX_CELLS = 2 * NOALLOC_MAX_POINTS + 512;  // the dense-grid budget of grid.rs
constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t OFF_PKEY = 0;
constexpr size_t OFF_KEYS = OFF_PKEY + align256(8 * (size_t)NOALLOC_MAX_POINTS);
constexpr size_t OFF_INDICES = OFF_KEYS + align256(8 * (size_t)NOALLOC_MAX_POINTS);
constexpr size_t OFF_CELL_START = OFF_INDICES + align256(4 * (size_t)NOALLOC_MAX_POINTS);
constexpr size_t OFF_CURSOR = OFF_CELL_START + align256(4 * ((size_t)NOALLOC_MAX_CELLS + 1));
constexpr size_t NOALLOC_SCRATCH_BYTES = OFF_CURSOR + align256(4 * ((size_t)NOALLOC_MAX_CELLS + 1));

// The grid scratch of every call on this device (file scope, fixed size).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

__global__ void __launch_bounds__(512) neighbor_lists_noalloc_kernel(const float2* __restrict__ xy, uint32_t n,
                                                                     float h, unsigned char* scratch, uint32_t* off,
                                                                     uint32_t* nbrs, uint32_t cap,
                                                                     uint32_t* n_edges_out, uint32_t* status_out) {
  __shared__ GridHdr hdr;
  __shared__ uint32_t n_edges;  // edges written (0 when cap is too small)
  __shared__ uint32_t err;
  GridBuf gb;
  gb.pkey = reinterpret_cast<int2*>(scratch + OFF_PKEY);
  gb.keys = reinterpret_cast<int2*>(scratch + OFF_KEYS);
  gb.indices = reinterpret_cast<uint32_t*>(scratch + OFF_INDICES);
  gb.cell_start = reinterpret_cast<uint32_t*>(scratch + OFF_CELL_START);
  gb.cursor = reinterpret_cast<uint32_t*>(scratch + OFF_CURSOR);
  gb.cap_points = NOALLOC_MAX_POINTS;
  gb.cap_cells = NOALLOC_MAX_CELLS;
  if (threadIdx.x == 0) err = 0;
  __syncthreads();
  grid_build(xy, n, h, gb, hdr, &err);
  build_neighbor_lists(xy, n, h, hdr, gb, off, nbrs, cap, &err, &n_edges);
  __syncthreads();
  if (threadIdx.x == 0) {
    *n_edges_out = off[n];  // the full count, also when it exceeds cap (n_edges is 0 then)
    *status_out = err;
  }
}

// Per-device address of the scratch, resolved once with that device current.
constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[MAX_DEVICES] = {};

int scratch_for_current_device(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_global_error(MG_ERR_NO_DEVICE, cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return set_global_error(MG_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return set_global_error(MG_ERR_CUDA, cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return MG_OK;
}

}  // namespace

}  // namespace mg

extern "C" int mg_neighbor_lists_noalloc(const float* xy_dev, uint32_t n, float h, uint32_t* offsets_dev,
                                         uint32_t* nbrs_dev, uint32_t cap, uint32_t* n_edges_dev,
                                         uint32_t* status_dev, void* stream) {
  using namespace mg;
  if (n > NOALLOC_MAX_POINTS) {
    char msg[160];
    snprintf(msg, sizeof(msg), "%u points exceed the no-allocation limit of %u points per call", n,
             NOALLOC_MAX_POINTS);
    return set_global_error(MG_ERR_CAPACITY, msg);
  }
  if (!(h > 0.0f) || !std::isfinite(h)) return set_global_error(MG_ERR_ARG, "h must be positive and finite");
  if ((n && !xy_dev) || !offsets_dev || (cap && !nbrs_dev) || !n_edges_dev || !status_dev)
    return set_global_error(MG_ERR_ARG, "null device pointer");
  void* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  neighbor_lists_noalloc_kernel<<<1, 512, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(xy_dev), n, h, static_cast<unsigned char*>(scratch), offsets_dev, nbrs_dev, cap,
      n_edges_dev, status_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_global_error(MG_ERR_CUDA, cudaGetErrorString(e));
  return MG_OK;
}
