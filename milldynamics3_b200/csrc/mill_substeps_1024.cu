// The mill sub-step kernel instantiated for blocks of up to 1024 threads.
#include "mill_substeps.cuh"

namespace mg {

cudaError_t launch_substeps_1024(const MillDev* mills, uint32_t n_mills, StepUniform* uni, const SubAngles* angles,
                               uint32_t n_sub, const uint32_t* n_sub_of, uint32_t threads, size_t smem_bytes,
                               cudaStream_t stream, uint32_t mill_blocks, const uint32_t* block_mill) {
  return launch_substeps_impl<1024>(mills, n_mills, uni, angles, n_sub, n_sub_of, threads, smem_bytes, stream,
                                  mill_blocks, block_mill);
}

}  // namespace mg
