// Vector-tile kernels (KIND_VTILE, vtile.cuh) and their dispatch.
#include <cuda_runtime.h>

#include "launch.h"
#include "vtile.cuh"

namespace hptt_b200 {

using namespace dev;

namespace {

// One CTA per tile, 256 or 512 threads.  Two register budgets, picked per
// plan by the tuner (HpttTile::vj): eight 16-byte vectors per thread and
// phase at 64 registers (1024 resident threads per SM), or four at 32
// registers (2048; a few variants spill up to 12 bytes).  Measured per shape,
// neither wins everywhere: the f32 2D update {35014, 1428} ran 6.1 TB/s with
// four and 6.0 with eight, the rank-6 {30, 4, 34, 42, 29, 10} copy 5.0 and 5.1.
// Update tiles of the four-vector build can also read their B windows before
// the A loads (PRE, HpttTile::vpre), with the eight-vector build's budget.
template <typename E, int MODE, bool UPD, typename OffT, bool LX, bool LY, int JV, bool PRE>
__global__ void __launch_bounds__(512, (JV == 8 || PRE) ? 2 : 4)
    k_vtile(const __grid_constant__ HpttArgs args) {
  // programmatic dependent launch: as in k_tile (kernels.cu)
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  extern __shared__ __align__(16) unsigned char smem[];
  const Scal sc{args.alpha[0], args.alpha[1], args.beta[0], args.beta[1]};
  const Op<E, MODE, UPD> op(sc);
  vtile_one<E, MODE, UPD, OffT, LX, LY, JV, PRE>(args.p, args.t, static_cast<const E *>(args.A),
                                            static_cast<E *>(args.B),
                                            static_cast<const unsigned char *>(args.tables), op,
                                            reinterpret_cast<E *>(smem), blockIdx.x);
}

// 64-bit offsets read both sides from the tables; 32-bit offsets compute a
// single-dim side as q * stride.
template <typename E, int MODE, bool UPD, int JV, bool PRE>
const void *pick_side(const HpttTile &t) {
  if (t.big_offsets)
    return reinterpret_cast<const void *>(&k_vtile<E, MODE, UPD, int64_t, false, false, JV, PRE>);
  const bool lx = t.nx <= 1, ly = t.ny <= 1;
  if (lx && ly)
    return reinterpret_cast<const void *>(&k_vtile<E, MODE, UPD, uint32_t, true, true, JV, PRE>);
  if (lx)
    return reinterpret_cast<const void *>(&k_vtile<E, MODE, UPD, uint32_t, true, false, JV, PRE>);
  if (ly)
    return reinterpret_cast<const void *>(&k_vtile<E, MODE, UPD, uint32_t, false, true, JV, PRE>);
  return reinterpret_cast<const void *>(&k_vtile<E, MODE, UPD, uint32_t, false, false, JV, PRE>);
}

template <typename E, int MODE, bool UPD>
const void *pick_shape(const HpttTile &t) {
  if (t.vj == 4) {
    if constexpr (UPD)
      if (t.vpre) return pick_side<E, MODE, UPD, 4, true>(t);
    return pick_side<E, MODE, UPD, 4, false>(t);
  }
  return pick_side<E, MODE, UPD, 8, false>(t);
}

}  // namespace

const void *vtile_kernel_for(const HpttArgs &a) {
  const bool upd = a.update != 0;
  const bool copy = a.mode == MODE_COPY && !upd;
  const HpttTile &t = a.t;
  switch (a.p.dtype) {
    case DT_F32:
      if (copy) return pick_shape<unsigned int, MODE_COPY, false>(t);
      if (a.mode == MODE_CPLX) return nullptr;
      return upd ? pick_shape<float, MODE_REAL, true>(t) : pick_shape<float, MODE_REAL, false>(t);
    case DT_F64:
      if (copy) return pick_shape<unsigned long long, MODE_COPY, false>(t);
      if (a.mode == MODE_CPLX) return nullptr;
      return upd ? pick_shape<double, MODE_REAL, true>(t) : pick_shape<double, MODE_REAL, false>(t);
    case DT_C64:
      if (copy) return pick_shape<unsigned long long, MODE_COPY, false>(t);
      if (a.mode == MODE_CPLX)
        return upd ? pick_shape<float2, MODE_CPLX, true>(t) : pick_shape<float2, MODE_CPLX, false>(t);
      return upd ? pick_shape<float2, MODE_REAL, true>(t) : pick_shape<float2, MODE_REAL, false>(t);
    default:
      return nullptr;  // 16-byte elements already move as 16-byte accesses
  }
}

}  // namespace hptt_b200
