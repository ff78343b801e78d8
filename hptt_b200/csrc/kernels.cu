// Single-transpose kernels and their host launchers.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.h"

namespace hptt_b200 {

using namespace dev;

namespace {

// Threads per CTA: 256 or 512 (HpttTile::nt; the planner's TileParams.nt).
constexpr int kMaxNT = 512;

// One CTA per tile.  The arguments live in the parameter space
// (__grid_constant__) and are read through a const reference.  Register
// budgets, stated for 512-thread CTAs (twice as many of 256 threads): 2048
// resident threads per SM for 4-byte copy/scale tiles (32 registers;
// measured +0.3 % over the sweep, up to +8 % on short-run shapes), 1536 for
// wider elements (the shared-memory limit at 32 KB a tile; at 32 registers
// they spill), 1024 when B is read too.
// Programmatic dependent launch: every launch may begin while the previous
// kernel on its stream is still running.  Each CTA first waits until that
// kernel has completed and its memory is visible (griddepcontrol.wait), so
// no global access moves ahead of it; only the launch and the CTA prologue
// overlap.  Each CTA then lets the next launch begin (it starts once every
// CTA of this grid has reached this point, i.e. during the last wave).  Both
// are no-ops when the launch was not made programmatic.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <typename E, int MODE, bool UPD, typename OffT, bool LX, bool LY>
__global__ void __launch_bounds__(kMaxNT, UPD ? 2 : (sizeof(E) <= 4 ? 4 : 3))
    k_tile(const __grid_constant__ HpttArgs args) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char smem[];
  const Scal sc{args.alpha[0], args.alpha[1], args.beta[0], args.beta[1]};
  const Op<E, MODE, UPD> op(sc);
  tile_one<E, MODE, UPD, OffT, LX, LY>(args.p, args.t, static_cast<const E *>(args.A),
                                       static_cast<E *>(args.B),
                                       static_cast<const unsigned char *>(args.tables), op,
                                       reinterpret_cast<E *>(smem), blockIdx.x);
}

template <typename E, int MODE, bool UPD, typename OffT, int VEC>
__global__ void __launch_bounds__(kMaxNT) k_rows(const __grid_constant__ HpttArgs args) {
  pdl_enter();
  const Scal sc{args.alpha[0], args.alpha[1], args.beta[0], args.beta[1]};
  const Op<E, MODE, UPD> op(sc);
  rows_one<E, MODE, UPD, OffT, VEC>(args.p, args.t, static_cast<const E *>(args.A),
                                    static_cast<E *>(args.B),
                                    static_cast<const unsigned char *>(args.tables), op,
                                    blockIdx.x);
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
// 64-bit table offsets only on the general path; single-dim sides compute
// their offsets in 64 bits anyway.
template <typename E, int MODE, bool UPD, typename OffT>
const void *pick_tile(const HpttTile &t) {
  if (sizeof(OffT) == 8) return reinterpret_cast<const void *>(&k_tile<E, MODE, UPD, int64_t, false, false>);
  const bool lx = t.nx <= 1, ly = t.ny <= 1;
  if (lx && ly) return reinterpret_cast<const void *>(&k_tile<E, MODE, UPD, uint32_t, true, true>);
  if (lx) return reinterpret_cast<const void *>(&k_tile<E, MODE, UPD, uint32_t, true, false>);
  if (ly) return reinterpret_cast<const void *>(&k_tile<E, MODE, UPD, uint32_t, false, true>);
  return reinterpret_cast<const void *>(&k_tile<E, MODE, UPD, uint32_t, false, false>);
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
    return t.big_offsets ? pick_tile<E, MODE, UPD, int64_t>(t) : pick_tile<E, MODE, UPD, uint32_t>(t);
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
  if (a.t.kind == KIND_VTILE) return vtile_kernel_for(a);
  if (a.t.kind == KIND_TTILE) return ttile_kernel_for(a);
  const bool upd = a.update != 0;
  switch (a.p.dtype) {
    case DT_F32: return pick_mode<float, unsigned int>(a.mode, upd, a.t, vec);
    case DT_F64: return pick_mode<double, unsigned long long>(a.mode, upd, a.t, vec);
    case DT_C64: return pick_mode_cplx<float2, unsigned long long>(a.mode, upd, a.t, vec);
    case DT_C128: return pick_mode_cplx<double2, uint4>(a.mode, upd, a.t, vec);
    default: return nullptr;
  }
}

int kernel_threads() { return kMaxNT; }

cudaError_t launch_single(const HpttArgs &a, int vec, int grid, cudaStream_t stream) {
  if (a.t.kind == KIND_TTILE) return launch_ttile(a, grid, stream);
  (void)grid;  // one CTA per tile
  const void *fn = kernel_for(a, vec);
  if (!fn) return cudaErrorInvalidValue;
  if (a.t.num_tiles == 0) return cudaSuccess;
  void *params[] = {const_cast<HpttArgs *>(&a)};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.t.num_tiles);
  cfg.blockDim = dim3(a.t.nt);
  cfg.dynamicSmemBytes = static_cast<size_t>(a.t.smem_bytes);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, params);
}

cudaError_t occupancy(const HpttArgs &a, int vec, int *ctas_per_sm) {
  const void *fn = kernel_for(a, vec);
  if (!fn) return cudaErrorInvalidValue;
  // One kernel serves many plans: always allow the device's opt-in maximum,
  // so a later plan with a smaller tile cannot lower the limit under an
  // earlier one.
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (a.t.smem_bytes > optin) return cudaErrorInvalidValue;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, a.t.nt,
                                                       static_cast<size_t>(a.t.smem_bytes));
}

}  // namespace hptt_b200
