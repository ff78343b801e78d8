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
// Thread mapping (vt_pos): a warp covers 8 consecutive window slots of 4
// rows (load) or of 4 columns (store), so every global access of a warp is
// four 128-byte runs; a thread walks every eighth slot of its rows or
// columns, at most JV (4 or 8, HpttTile::vj) vectors per phase.  The host
// picks the row pitch LD that minimises shared-memory bank conflicts of
// exactly these accesses (vtile_bank_cost).
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

// Thread `tid` -> (first window slot k of its lines, first line r0) of
// either phase: a warp holds 8 consecutive slots of 4 lines (4 * 128 bytes
// per access); a thread takes slots k, k + 8, ... of each of its lines, and
// lines r0 + j * (nt / 8).  So a line's offset and window shift are worked
// out once per thread and line, not once per vector.
struct VtPos {
  int k, r0;
};

HPTT_HD inline VtPos vt_pos(int tid) {
  VtPos p;
  p.k = tid & 7;
  p.r0 = ((tid >> 5) << 2) | ((tid >> 3) & 3);
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

// Load phase: rows of A into shared memory.  Thread (k, r0) reads window
// slots k + 8 g (g < G, the row's number of 8-slot groups) of rows
// r0 + j * R1, at most JV vectors in all.  A
// row's offset steps by R1 * sya (one Y dim) or comes from the table; its
// window shift is (shift of the tile origin + row offset) mod V.  Every
// window of a row below limY goes to shared memory whole: a window that was
// not read (it starts at or past limX) lands in the row's padding.
template <typename E, typename OffT, bool LY, int LG, int JV>
__device__ __forceinline__ void vt_load(const HpttTile &T, const E *__restrict__ a0,
                                        const OffT *__restrict__ tabY, E *sm, int limX,
                                        int limY) {
  constexpr int V = 16 / sizeof(E);
  constexpr int G = 1 << LG;
  using VecT = Vec<E, V>;
  const VtPos ps = vt_pos(threadIdx.x);
  const int xk = ps.k * V;
  const int R1 = T.R1;
  const int s0 = vt_shift(a0);
  const int LD = T.LD;
  with_trip_count<JV / G>(T.J1, [&](auto nn) {
    constexpr int N = decltype(nn)::value;
    VecT v[N][G];
    int sh[N];
    OffT off = LY ? static_cast<OffT>(ps.r0) * static_cast<OffT>(T.sya) : OffT(0);
    const OffT stepA = LY ? static_cast<OffT>(R1) * static_cast<OffT>(T.sya) : OffT(0);
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const int y = ps.r0 + j * R1;
      if (!LY) off = tabY[min(y, T.TY - 1)];
      const int s = (s0 + static_cast<int>(off)) & (V - 1);
      sh[j] = y < limY ? s : -1;
      const E *w = a0 + static_cast<int64_t>(off) + (xk - s);
#pragma unroll
      for (int g = 0; g < G; ++g)
        if (sh[j] >= 0 && xk + 8 * V * g - s < limX) v[j][g] = ld_vec<E, V>(w + 8 * V * g);
      if (LY) off += stepA;
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      if (sh[j] >= 0) {
        E *d = sm + (ps.r0 + j * R1) * LD + xk - sh[j];
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
          for (int i = 0; i < V; ++i) d[8 * V * g + i] = v[j][g].v[i];
      }
    }
  });
}

// Column x's B offset and window shift, -1 when the column is outside the
// tile (shared by the store phase and the early B reads).
template <typename E, typename OffT, bool LX>
__device__ __forceinline__ int vt_column(const HpttTile &T, const OffT *__restrict__ tabX,
                                         int x, int t0, int limX, OffT &off) {
  constexpr int V = 16 / sizeof(E);
  off = LX ? static_cast<OffT>(x) * static_cast<OffT>(T.sxb) : tabX[min(x, T.TX - 1)];
  const int t = (t0 + static_cast<int>(off)) & (V - 1);
  return x < limX ? t : -1;
}

// The store phase's B windows, read before the load phase so they are in
// flight together with the A loads (update tiles, HpttTile::vpre): slot g of
// the thread's column j lands in bv[j * G + g].
template <typename E, typename OffT, bool LX, int LG, int JV>
__device__ __forceinline__ void vt_bread(const HpttTile &T, const E *__restrict__ b0,
                                         const OffT *__restrict__ tabX,
                                         Vec<E, 16 / sizeof(E)> *bv, int limX, int limY) {
  constexpr int V = 16 / sizeof(E);
  constexpr int G = 1 << LG;
  const VtPos ps = vt_pos(threadIdx.x);
  const int yk = ps.k * V;
  const int t0 = vt_shift(b0);
  with_trip_count<JV / G>(T.J2, [&](auto nn) {
    constexpr int N = decltype(nn)::value;
#pragma unroll
    for (int j = 0; j < N; ++j) {
      OffT off;
      const int t = vt_column<E, OffT, LX>(T, tabX, ps.r0 + j * T.R2, t0, limX, off);
      const E *w = b0 + static_cast<int64_t>(off) + (yk - t);
#pragma unroll
      for (int g = 0; g < G; ++g)
        if (t >= 0 && yk + 8 * V * g - t < limY) bv[j * G + g] = ld_vec_rw<E, V>(w + 8 * V * g);
    }
  });
}

// Store phase: columns of B from shared memory.  Thread (k, c0) writes window
// slots k + 8 g of columns c0 + j * R2; slot element i is y = V (k + 8 g) - t
// + i, t the column's window shift.  When B is read, all of the thread's B
// windows are read before the first store: here (PRE off) or, with PRE,
// before the load phase (vt_bread, passed in as `pre`).
template <typename E, int MODE, bool UPD, typename OffT, bool LX, int LG, int JV, bool PRE>
__device__ __forceinline__ void vt_store(const HpttTile &T, E *__restrict__ b0,
                                         const OffT *__restrict__ tabX, const E *sm,
                                         const Op<E, MODE, UPD> &op, int limX, int limY,
                                         const Vec<E, 16 / sizeof(E)> *pre) {
  constexpr int V = 16 / sizeof(E);
  constexpr int G = 1 << LG;
  using VecT = Vec<E, V>;
  const VtPos ps = vt_pos(threadIdx.x);
  const int yk = ps.k * V;
  const int R2 = T.R2;
  const int t0 = vt_shift(b0);
  const int LD = T.LD;
  with_trip_count<JV / G>(T.J2, [&](auto nn) {
    constexpr int N = decltype(nn)::value;
    // column j's offset and window shift (-1: outside the tile)
    auto column = [&](int j, OffT &off) -> int {
      return vt_column<E, OffT, LX>(T, tabX, ps.r0 + j * R2, t0, limX, off);
    };
    VecT bv[UPD && !PRE ? N : 1][UPD && !PRE ? G : 1];
    if (UPD && !PRE) {
#pragma unroll
      for (int j = 0; j < N; ++j) {
        OffT off;
        const int t = column(j, off);
        const E *w = b0 + static_cast<int64_t>(off) + (yk - t);
#pragma unroll
        for (int g = 0; g < G; ++g)
          if (t >= 0 && yk + 8 * V * g - t < limY)
            bv[UPD && !PRE ? j : 0][UPD && !PRE ? g : 0] = ld_vec_rw<E, V>(w + 8 * V * g);
      }
    }
#pragma unroll
    for (int j = 0; j < N; ++j) {
      OffT off;
      const int t = column(j, off);
      if (t < 0) continue;
      const E *s = sm + (yk - t) * LD + ps.r0 + j * R2;
      E *w = b0 + static_cast<int64_t>(off) + (yk - t);
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int y0 = yk + 8 * V * g - t;
        if (y0 >= limY) continue;
        VecT r;
#pragma unroll
        for (int i = 0; i < V; ++i) {
          const E a = s[(8 * V * g + i) * LD];
          const E b = !UPD ? a : (PRE ? pre[j * G + g].v[i] : bv[PRE ? 0 : j][PRE ? 0 : g].v[i]);
          r.v[i] = op(a, b);
        }
        E *dst = w + 8 * V * g;
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

template <typename E, int MODE, bool UPD, typename OffT, bool LX, bool LY, int JV, bool PRE>
__device__ __forceinline__ void vtile_one(const HpttProblem &P, const HpttTile &T,
                                          const E *__restrict__ A, E *__restrict__ B,
                                          const unsigned char *__restrict__ tables,
                                          const Op<E, MODE, UPD> &op, E *sdata,
                                          uint32_t tile) {
  constexpr int V = 16 / sizeof(E);
  static_assert(sizeof(Vec<E, V>) == 16, "16-byte vectors");
  const TileOrigin o = tile_origin(P, T, tile);
  const int limX = vt_lim_x(T, o), limY = vt_lim_y(T, o);
  E *sm = sdata + (V - 1) * (T.LD + 1);
  const OffT *__restrict__ tabY = reinterpret_cast<const OffT *>(tables);
  const OffT *__restrict__ tabX = reinterpret_cast<const OffT *>(tables + T.tab2_off);
  const E *a0 = A + o.bA;
  static_assert(JV == 4 || JV == 8, "4 or 8 vectors per thread");
  static_assert(!PRE || UPD, "early B reads for update tiles only");
  E *b0 = B + o.bB;
  Vec<E, V> bpre[PRE ? JV : 1];
  if (PRE) {
    if (T.vly == 0)
      vt_bread<E, OffT, LX, 0, JV>(T, b0, tabX, bpre, limX, limY);
    else if (T.vly == 1)
      vt_bread<E, OffT, LX, 1, JV>(T, b0, tabX, bpre, limX, limY);
    else
      vt_bread<E, OffT, LX, 2, JV>(T, b0, tabX, bpre, limX, limY);
  }
  if (T.vlx == 0)
    vt_load<E, OffT, LY, 0, JV>(T, a0, tabY, sm, limX, limY);
  else if (T.vlx == 1)
    vt_load<E, OffT, LY, 1, JV>(T, a0, tabY, sm, limX, limY);
  else
    vt_load<E, OffT, LY, 2, JV>(T, a0, tabY, sm, limX, limY);
  __syncthreads();
  if (T.vly == 0)
    vt_store<E, MODE, UPD, OffT, LX, 0, JV, PRE>(T, b0, tabX, sm, op, limX, limY, bpre);
  else if (T.vly == 1)
    vt_store<E, MODE, UPD, OffT, LX, 1, JV, PRE>(T, b0, tabX, sm, op, limX, limY, bpre);
  else
    vt_store<E, MODE, UPD, OffT, LX, 2, JV, PRE>(T, b0, tabX, sm, op, limX, limY, bpre);
}

}  // namespace dev
}  // namespace hptt_b200
