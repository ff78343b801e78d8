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

// The TMA-tile kernel (KIND_TTILE) for these arguments, or null.
const void *ttile_kernel_for(const HpttArgs &a);

// Enqueue one KIND_TTILE transpose: encodes the tensor maps of A and B
// (16-byte aligned bases required: cudaErrorMisalignedAddress otherwise) and
// launches with them, one CTA per tile or (persistent form, HpttTile::ts)
// min(grid, tiles) CTAs.
cudaError_t launch_ttile(const HpttArgs &a, int grid, cudaStream_t stream);

// Most threads per CTA the single-transpose kernels are compiled for.
int kernel_threads();

// Enqueue one transpose: one CTA per tile, except the persistent TMA tile,
// whose `grid` CTAs loop over the tiles.
cudaError_t launch_single(const HpttArgs &a, int vec, int grid, cudaStream_t stream);

// Resident CTAs per SM for this launch shape (also raises the dynamic
// shared-memory limit of the kernel when needed).
cudaError_t occupancy(const HpttArgs &a, int vec, int *ctas_per_sm);

}  // namespace hptt_b200
