// Single-transpose kernels and their host launchers.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.h"

namespace hptt_b200 {

using namespace dev;

namespace {

constexpr int kNT = 256;

// Copy the launch arguments into shared memory with compile-time-indexed
// word moves, so the kernels index dims dynamically from shared memory
// rather than from the parameter space.
__device__ __forceinline__ void stage_args(const HpttArgs &src, HpttArgs *dst) {
  static_assert(sizeof(HpttArgs) % 8 == 0, "HpttArgs must be 8-byte sized");
  constexpr int kWords = sizeof(HpttArgs) / 8;
  const uint64_t *s = reinterpret_cast<const uint64_t *>(&src);
  uint64_t *d = reinterpret_cast<uint64_t *>(dst);
#pragma unroll
  for (int i = 0; i < kWords; i += 32) {
    const int w = i + static_cast<int>(threadIdx.x % 32);
    if (threadIdx.x < 32 && w < kWords) d[w] = s[w];
  }
}

template <typename E, int MODE, bool UPD, typename OffT>
__global__ void __launch_bounds__(kNT, 3) k_tile(const __grid_constant__ HpttArgs args) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ HpttArgs sa;
  stage_args(args, &sa);
  __syncthreads();
  const HpttProblem &P = sa.p;
  const HpttTile &T = sa.t;
  E *sdata = reinterpret_cast<E *>(smem);
  const int data_bytes = align16(T.TY * T.LD * static_cast<int>(sizeof(E)));
  OffT *tInY = reinterpret_cast<OffT *>(smem + data_bytes);
  OffT *tOutX = tInY + T.TY;
  int *tCy = reinterpret_cast<int *>(tOutX + T.TX);
  int *tCx = tCy + T.TY;
  tile_tables<OffT>(P, T, tInY, tCy, tOutX, tCx, threadIdx.x, blockDim.x);
  const TileThread<OffT> s = tile_thread<OffT>(P, T, threadIdx.x);
  const Scal sc{sa.alpha[0], sa.alpha[1], sa.beta[0], sa.beta[1]};
  const Op<E, MODE, UPD> op(sc);
  const E *A = static_cast<const E *>(sa.A);
  E *B = static_cast<E *>(sa.B);
  __syncthreads();
  for (uint32_t tile = blockIdx.x; tile < T.num_tiles; tile += gridDim.x) {
    const TileOrigin o = tile_origin(P, T, tile);
    tile_body<E, MODE, UPD, OffT>(T, A, B, op, s, o, sdata, tInY, tCy, tOutX, tCx);
  }
}

template <typename E, int MODE, bool UPD, typename OffT, int VEC>
__global__ void __launch_bounds__(kNT, 2) k_rows(const __grid_constant__ HpttArgs args) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ HpttArgs sa;
  stage_args(args, &sa);
  __syncthreads();
  const HpttProblem &P = sa.p;
  const HpttTile &T = sa.t;
  OffT *tInY = reinterpret_cast<OffT *>(smem);
  OffT *tOutY = tInY + T.TY;
  int *tCy = reinterpret_cast<int *>(tOutY + T.TY);
  rows_tables<OffT>(P, T, tInY, tOutY, tCy, threadIdx.x, blockDim.x);
  const RowThread<OffT> s = rows_thread<OffT>(T, threadIdx.x);
  const Scal sc{sa.alpha[0], sa.alpha[1], sa.beta[0], sa.beta[1]};
  const Op<E, MODE, UPD> op(sc);
  const E *A = static_cast<const E *>(sa.A);
  E *B = static_cast<E *>(sa.B);
  __syncthreads();
  for (uint32_t tile = blockIdx.x; tile < T.num_tiles; tile += gridDim.x) {
    const TileOrigin o = tile_origin(P, T, tile);
    rows_body<E, MODE, UPD, OffT, VEC>(P, T, A, B, op, s, o, tInY, tOutY, tCy);
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
template <typename E, int MODE, bool UPD, typename OffT>
const void *pick_tile() {
  return reinterpret_cast<const void *>(&k_tile<E, MODE, UPD, OffT>);
}

template <typename E, int MODE, bool UPD, typename OffT>
const void *pick_rows(int vec_bytes) {
  constexpr int S = sizeof(E);
  switch (vec_bytes / S) {
    case 4: if (S == 4) return reinterpret_cast<const void *>(&k_rows<E, MODE, UPD, OffT, (S == 4 ? 4 : 1)>); break;
    case 2: if (S <= 8) return reinterpret_cast<const void *>(&k_rows<E, MODE, UPD, OffT, (S <= 8 ? 2 : 1)>); break;
    default: break;
  }
  return reinterpret_cast<const void *>(&k_rows<E, MODE, UPD, OffT, 1>);
}

template <typename E, int MODE, bool UPD>
const void *pick_off(const HpttTile &t, int vec) {
  const int vb = vec * static_cast<int>(sizeof(E));
  if (t.kind == KIND_TILE)
    return t.big_offsets ? pick_tile<E, MODE, UPD, int64_t>() : pick_tile<E, MODE, UPD, uint32_t>();
  return t.big_offsets ? pick_rows<E, MODE, UPD, int64_t>(vb) : pick_rows<E, MODE, UPD, uint32_t>(vb);
}

template <typename E, typename ER>
const void *pick_mode(int mode, bool upd, const HpttTile &t, int vec) {
  // ER: raw storage of the same width, used for bit copies
  if (mode == MODE_COPY && !upd) return pick_off<ER, MODE_COPY, false>(t, vec);
  if (mode == MODE_CPLX) return nullptr;
  return upd ? pick_off<E, MODE_REAL, true>(t, vec) : pick_off<E, MODE_REAL, false>(t, vec);
}

template <typename E, typename ER>
const void *pick_mode_cplx(int mode, bool upd, const HpttTile &t, int vec) {
  if (mode == MODE_COPY && !upd) return pick_off<ER, MODE_COPY, false>(t, vec);
  if (mode == MODE_CPLX)
    return upd ? pick_off<E, MODE_CPLX, true>(t, vec) : pick_off<E, MODE_CPLX, false>(t, vec);
  return upd ? pick_off<E, MODE_REAL, true>(t, vec) : pick_off<E, MODE_REAL, false>(t, vec);
}

}  // namespace

const void *kernel_for(const HpttArgs &a, int vec) {
  const bool upd = a.update != 0;
  switch (a.p.dtype) {
    case DT_F32: return pick_mode<float, unsigned int>(a.mode, upd, a.t, vec);
    case DT_F64: return pick_mode<double, unsigned long long>(a.mode, upd, a.t, vec);
    case DT_C64: return pick_mode_cplx<float2, unsigned long long>(a.mode, upd, a.t, vec);
    case DT_C128: return pick_mode_cplx<double2, uint4>(a.mode, upd, a.t, vec);
    default: return nullptr;
  }
}

int kernel_threads() { return kNT; }

cudaError_t launch_single(const HpttArgs &a, int vec, int grid, cudaStream_t stream) {
  const void *fn = kernel_for(a, vec);
  if (!fn) return cudaErrorInvalidValue;
  if (a.t.num_tiles == 0) return cudaSuccess;
  void *params[] = {const_cast<HpttArgs *>(&a)};
  return cudaLaunchKernel(fn, dim3(grid), dim3(a.t.nt), params,
                          static_cast<size_t>(a.t.smem_bytes), stream);
}

cudaError_t occupancy(const HpttArgs &a, int vec, int *ctas_per_sm) {
  const void *fn = kernel_for(a, vec);
  if (!fn) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       a.t.smem_bytes > 48 * 1024 ? a.t.smem_bytes : 48 * 1024);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, a.t.nt,
                                                       static_cast<size_t>(a.t.smem_bytes));
}

}  // namespace hptt_b200
