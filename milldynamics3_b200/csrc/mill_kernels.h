// Host-visible launch wrappers of mill_kernels.cu.
#pragma once

#include "mill_common.cuh"

namespace mg {

// Runs n_sub coupled sub-steps on each of n_mills mills (one block per mill). uni holds one
// StepUniform per mill; angles holds n_mills * n_sub SubAngles, mill-major.
cudaError_t launch_substeps(const MillDev* mills, uint32_t n_mills, StepUniform* uni, const SubAngles* angles,
                            uint32_t n_sub, uint32_t threads, cudaStream_t stream);
// Grid-stage probe over the descriptor's fx[0..nf): mode 0 grid, 1 candidate pairs, 2 neighbours.
cudaError_t launch_probe(const MillDev* mill, float cell, int mode, uint32_t* result, cudaStream_t stream);

}  // namespace mg
