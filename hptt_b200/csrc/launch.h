// Host-side entry points into the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include "desc.h"

namespace hptt_b200 {

// Kernel function for these arguments; vec = elements per access for
// KIND_ROWS (1 when the pointers are not aligned for the planned vector).
const void *kernel_for(const HpttArgs &a, int vec);

// The vector-tile kernel (KIND_VTILE) for these arguments, or null.
const void *vtile_kernel_for(const HpttArgs &a);

// Most threads per CTA the single-transpose kernels are compiled for.
int kernel_threads();

// Enqueue one transpose.  `grid` CTAs loop over the tiles.
cudaError_t launch_single(const HpttArgs &a, int vec, int grid, cudaStream_t stream);

// Resident CTAs per SM for this launch shape (also raises the dynamic
// shared-memory limit of the kernel when needed).
cudaError_t occupancy(const HpttArgs &a, int vec, int *ctas_per_sm);

}  // namespace hptt_b200
