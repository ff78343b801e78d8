// sm_100a vector tile: B = alpha * A(perm) + beta * B with 16-byte global
// accesses on both sides of the shared-memory transpose.
//
// Shape (KIND_VTILE, planned by choose_tile): the tile's X side is input
// dims 0..nx-1, all full but the last, so the X coordinates of one row are
// ONE contiguous run of A (x is the element offset from the row start); its
// Y side is output dims 0..ny-1, all full but the last, so the Y coordinates
// of one column are one contiguous run of B.  Row y starts at A offset
// rowA(y) (y * stride for one Y dim, else the plan's table), column x at B
// offset colB(x).  Elements are 4 or 8 bytes; V = 16 / sizeof(E) per vector.
//
// Runs start anywhere: the extents are arbitrary, so most rows and columns
// are not 16-byte aligned.  The kernel works on the 16-byte-aligned windows
// that cover each run:
//   load phase   row y is read as aligned windows starting s(y) elements
//                before the row (s = row address / sizeof(E) mod V).  A
//                window that holds at least one element of the row is read
//                whole: its other elements share its 16-byte block with an
//                element of the tensor, so the read stays inside the
//                allocation's pages, and they are discarded (written to
//                shared-memory padding that no store reads).  All V elements
//                go to shared memory at their own column x (four 4-byte or
//                two 8-byte shared stores), so the store phase reads plain
//                (x, y) positions.
//   store phase  column x is written as aligned windows starting t(x)
//                elements before the column.  A window wholly inside the
//                column is one 16-byte store; the (at most two) windows at
//                the column's ends store only their elements inside it, one
//                by one.  When B is read, the B window is read whole first
//                (same 16-byte-block argument) and only its column's
//                elements are written back.
// Thread mapping: a warp covers 8 consecutive window slots of 4 rows (load)
// or of 4 columns (store): every global access of a warp is four 128-byte
// runs, and the host picks the row pitch LD that minimises shared-memory
// bank conflicts of exactly these accesses (vtile_bank_cost).
//
// This replaces the reference's 256-bit in-register micro kernels
// (src/arch/avx2/kernel_trans_avx2.cc:21-467) for shapes whose contiguous
// runs lie on both sides of the transpose.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "desc.h"
#include "kernels.cuh"
#include "ops.cuh"

namespace hptt_b200 {
namespace dev {

// Vector loads (rows) or stores (columns) a thread keeps in flight per phase.
HPTT_HD constexpr int hptt_vt_jmax() { return 8; }

// Thread `tid` -> (window slot k along a line, first line r0) of one phase;
// lines r0 + j * (nt >> (3 + lg)).  A warp holds 8 slots of 4 lines; a line
// has 8 << lg slots.
struct VtPos {
  int k, r0;
};

HPTT_HD inline VtPos vt_pos(int tid, int lg) {
  const int w = tid >> 5;
  VtPos p;
  p.k = (tid & 7) | ((w & ((1 << lg) - 1)) << 3);
  p.r0 = ((tid >> 3) & 3) | ((w >> lg) << 2);
  return p;
}

// Valid extents of this tile along the X run and the Y run: the chunked
// (last) dim of a side is the slowest in its run, so run position x is
// inside the tensor when x < px * remX.
HPTT_HD inline int vt_lim_x(const HpttTile &T, const TileOrigin &o) {
  return (T.xc >= 0 && o.remX < T.xce) ? T.px * o.remX : T.TX;
}

HPTT_HD inline int vt_lim_y(const HpttTile &T, const TileOrigin &o) {
  return (T.yc >= 0 && o.remY < T.yce) ? T.py * o.remY : T.TY;
}

// Shared memory: element (x, y) at (y + V - 1) * LD + (x + V - 1); rows and
// columns run from -(V - 1) so the windows' outside elements land in padding.
HPTT_HD constexpr int vt_pad(int esz) { return 16 / esz - 1; }

template <typename E, int V>
__device__ __forceinline__ void st_vec_cs(E *p, const Vec<E, V> &v) {
  uint4 r;
  memcpy(&r, &v, sizeof(r));
  __stcs(reinterpret_cast<uint4 *>(p), r);
}

template <typename E>
__device__ __forceinline__ int vt_shift(const E *p) {
  constexpr int V = 16 / sizeof(E);
  return static_cast<int>((reinterpret_cast<uintptr_t>(p) / sizeof(E)) & (V - 1));
}

template <typename E, int MODE, bool UPD, typename OffT, bool LX, bool LY>
__device__ __forceinline__ void vtile_one(const HpttProblem &P, const HpttTile &T,
                                          const E *__restrict__ A, E *__restrict__ B,
                                          const unsigned char *__restrict__ tables,
                                          const Op<E, MODE, UPD> &op, E *sdata,
                                          uint32_t tile) {
  constexpr int V = 16 / sizeof(E);
  constexpr int JV = hptt_vt_jmax();
  using VecT = Vec<E, V>;
  static_assert(sizeof(VecT) == 16, "16-byte vectors");
  const TileOrigin o = tile_origin(P, T, tile);
  const int limX = vt_lim_x(T, o), limY = vt_lim_y(T, o);
  const int LD = T.LD;
  E *sm = sdata + (V - 1) * (LD + 1);
  const OffT *__restrict__ tabY = reinterpret_cast<const OffT *>(tables);
  const OffT *__restrict__ tabX = reinterpret_cast<const OffT *>(tables + T.tab2_off);
  // ---- load phase: rows of A into shared memory ----
  // Thread (k, r0) reads window slot k of rows r0 + j * R1.  A row's offset
  // steps by R1 * sya (one Y dim) or comes from the table; its window shift
  // is (shift of the tile origin + row offset) mod V.
  {
    const VtPos ps = vt_pos(threadIdx.x, T.vlx);
    const int xk = ps.k * V;
    const int R1 = T.R1;
    const E *a0 = A + o.bA;
    const int s0 = vt_shift(a0);
    const OffT stepA = LY ? static_cast<OffT>(R1) * static_cast<OffT>(T.sya) : OffT(0);
    E *srow = sm + ps.r0 * LD + xk;
    const int sstep = R1 * LD;
    with_trip_count<JV>(T.J1, [&](auto nn) {
      constexpr int N = decltype(nn)::value;
      VecT v[N];
      int sh[N];
      OffT off = LY ? static_cast<OffT>(ps.r0) * static_cast<OffT>(T.sya) : OffT(0);
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const int y = ps.r0 + j * R1;
        if (!LY) off = tabY[min(y, T.TY - 1)];
        const int s = (s0 + static_cast<int>(off)) & (V - 1);
        sh[j] = (y < limY && xk - s < limX) ? s : -1;
        if (sh[j] >= 0) v[j] = ld_vec<E, V>(a0 + static_cast<int64_t>(off) + (xk - s));
        if (LY) off += stepA;
      }
#pragma unroll
      for (int j = 0; j < N; ++j) {
        if (sh[j] >= 0) {
          E *d = srow + j * sstep - sh[j];
#pragma unroll
          for (int i = 0; i < V; ++i) d[i] = v[j].v[i];
        }
      }
    });
  }
  __syncthreads();
  // ---- store phase: columns of B from shared memory ----
  // Thread (k, c0) writes window slot k of columns c0 + j * R2: element y of
  // the slot is y0 + i with y0 = V * k - t (t = the column's window shift).
  const VtPos ps = vt_pos(threadIdx.x, T.vly);
  const int yk = ps.k * V;
  const int R2 = T.R2;
  E *b0 = B + o.bB;
  const int t0 = vt_shift(b0);
  const E *scol = sm + yk * LD + ps.r0;
  with_trip_count<JV>(T.J2, [&](auto nn) {
    constexpr int N = decltype(nn)::value;
    // column j's offset and window shift (-1: nothing of it in this slot)
    auto column = [&](int j, OffT &off) -> int {
      const int x = ps.r0 + j * R2;
      off = LX ? static_cast<OffT>(x) * static_cast<OffT>(T.sxb) : tabX[min(x, T.TX - 1)];
      const int t = (t0 + static_cast<int>(off)) & (V - 1);
      return (x < limX && yk - t < limY) ? t : -1;
    };
    VecT bv[UPD ? N : 1];
    if (UPD) {
      // the B windows first, all in flight together
#pragma unroll
      for (int j = 0; j < N; ++j) {
        OffT off;
        const int t = column(j, off);
        if (t >= 0) bv[UPD ? j : 0] = ld_vec_rw<E, V>(b0 + static_cast<int64_t>(off) + (yk - t));
      }
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      OffT off;
      const int t = column(j, off);
      if (t >= 0) {
        const E *s = scol + j * R2 - t * LD;
        VecT r;
#pragma unroll
        for (int i = 0; i < V; ++i) {
          const E a = s[i * LD];
          r.v[i] = op(a, UPD ? bv[UPD ? j : 0].v[i] : a);
        }
        E *dst = b0 + static_cast<int64_t>(off) + (yk - t);
        const int y0 = yk - t;
        if (y0 >= 0 && y0 + V <= limY) {
          if (UPD)
            st_vec<E, V>(dst, r);
          else
            st_vec_cs<E, V>(dst, r);
        } else {
#pragma unroll
          for (int i = 0; i < V; ++i) {
            if (y0 + i >= 0 && y0 + i < limY) {
              if (UPD)
                dst[i] = r.v[i];
              else
                __stcs(dst + i, r.v[i]);
            }
          }
        }
      }
    }
  });
}

}  // namespace dev
}  // namespace hptt_b200
