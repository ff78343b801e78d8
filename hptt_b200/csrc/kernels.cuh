// sm_100a device code for B = alpha * A(perm) + beta * B.
//
// Replaces the reference's CPU macro/micro kernels
// (src/kernels/macro_kernel_trans.cc, src/arch/avx2/kernel_trans_avx2.cc):
//   tile_one  -- the in-register W x W transposes (kernel_trans_avx2.cc:21-467)
//                become one shared-memory tile per CTA that pairs the
//                input's stride-1 dims (X, with the shared block W) with the
//                output's (Y); reads and writes go in contiguous runs.
//                Ragged edges (the reference's scalar kernels,
//                macro_kernel_trans.cc:225-252) are integer compares in the
//                same pass.
//   rows_one  -- the shared-stride-1 linear kernel (kernel_trans_avx2.cc:480-530,
//                macro_kernel_trans.cc:181-195) becomes a vectorised
//                copy-scale over rows.
// Both fuse the beta * B read into the same pass.  Grids are one CTA per
// tile, so many small CTAs stay resident on every SM and keep enough loads
// in flight for HBM; a tile costs one mixed-radix decode of its index
// (multiply-high division), and every in-tile offset comes from small
// per-plan tables (L1-resident) computed on the host.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "desc.h"
#include "ops.cuh"

namespace hptt_b200 {
namespace dev {

// ---------------------------------------------------------------------------
// Memory helpers
// ---------------------------------------------------------------------------
// Fixed-width raw vector of VEC elements, moved as one 4/8/16-byte access.
template <typename E, int VEC>
struct alignas(sizeof(E) * VEC) Vec {
  E v[VEC];
};

template <int BYTES> struct RawT;
template <> struct RawT<4> { using T = unsigned int; };
template <> struct RawT<8> { using T = uint2; };
template <> struct RawT<16> { using T = uint4; };

template <typename E, int VEC>
__device__ __forceinline__ Vec<E, VEC> ld_vec(const E *p) {
  using R = typename RawT<sizeof(E) * VEC>::T;
  R r = __ldg(reinterpret_cast<const R *>(p));
  Vec<E, VEC> out;
  memcpy(&out, &r, sizeof(r));
  return out;
}

template <typename E, int VEC>
__device__ __forceinline__ Vec<E, VEC> ld_vec_rw(const E *p) {
  using R = typename RawT<sizeof(E) * VEC>::T;
  R r = *reinterpret_cast<const R *>(p);
  Vec<E, VEC> out;
  memcpy(&out, &r, sizeof(r));
  return out;
}

template <typename E, int VEC>
__device__ __forceinline__ void st_vec(E *p, const Vec<E, VEC> &v) {
  using R = typename RawT<sizeof(E) * VEC>::T;
  R r;
  memcpy(&r, &v, sizeof(r));
  *reinterpret_cast<R *>(p) = r;
}

// ---------------------------------------------------------------------------
// Tile geometry (host and device: the CPU replay in verify.cu uses it too)
// ---------------------------------------------------------------------------
HPTT_HD inline uint32_t umulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

struct TileOrigin {
  int64_t bA, bB;  // element offsets of the tile origin in A and B
  int remX;        // extent left along the chunked X (KIND_ROWS: W) dim, capped
  int remY;        // extent left along the chunked Y dim, capped
};

// Origin of tile `tile`: a mixed-radix decode over the grid levels, each
// level's steps folded by the planner (gsa, gsb, gn, gflag), so the loop --
// unrolled to the maximum rank -- reads every field at a static offset.
HPTT_HD inline TileOrigin tile_origin(const HpttProblem &P, const HpttTile &T,
                                      uint32_t tile) {
  (void)P;
  TileOrigin o;
  o.bA = 0;
  o.bB = 0;
  int64_t remX = 0x7fffffff, remY = 0x7fffffff;
  uint32_t rem = tile;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int g = 0; g < HPTT_MAX_RANK; ++g) {
    if (g < T.ng) {
      const uint32_t q = T.gmul[g] ? (umulhi32(rem, T.gmul[g]) >> T.gshr[g]) : rem;
      const uint32_t c = rem - q * T.gcnt[g];
      rem = q;
      o.bA += static_cast<int64_t>(c) * T.gsa[g];
      o.bB += static_cast<int64_t>(c) * T.gsb[g];
      const int64_t left = T.gn[g] - static_cast<int64_t>(c) * T.gstep[g];
      if (T.gflag[g] & 1) remX = left;
      if (T.gflag[g] & 2) remY = left;
    }
  }
  o.remX = static_cast<int>(remX < 0x7fffffff ? remX : 0x7fffffff);
  o.remY = static_cast<int>(remY < 0x7fffffff ? remY : 0x7fffffff);
  return o;
}

// Mixed-radix decomposition of a tile-local index over a list of dims.
template <typename OffT>
HPTT_HD inline OffT decompose(int idx, int nd, const int32_t *dims, const int32_t *ext,
                              const int64_t *stride) {
  OffT o = 0;
  for (int i = 0; i < nd; ++i) {
    const int c = idx % ext[i];
    idx /= ext[i];
    o += static_cast<OffT>(c) * static_cast<OffT>(stride[dims[i]]);
  }
  return o;
}

// Per-thread constants of the row copy.
struct RowThread {
  bool active;
  int e;   // vector index inside the row chunk
  int y0;
};

template <typename OffT>
HPTT_HD inline void rows_tables(const HpttProblem &P, const HpttTile &T, OffT *tInY,
                                OffT *tOutY, int tid, int nthreads) {
  for (int y = tid; y < T.TY; y += nthreads) {
    tInY[y] = decompose<OffT>(y, T.ny, T.yd, T.yt, P.sA);
    tOutY[y] = decompose<OffT>(y, T.ny, T.yd, T.yt, P.sB);
  }
}

HPTT_HD inline RowThread rows_thread(const HpttTile &T, int tid) {
  RowThread s;
  s.active = tid < T.R1 * T.RW;
  s.e = tid % T.RW;
  s.y0 = tid / T.RW;
  return s;
}

// Valid rows of a KIND_ROWS tile: the chunked Y dim is the last Y dim, so
// row y = rest + py * c is inside when y < remY * py.
HPTT_HD inline int rows_limit_y(const HpttTile &T, const TileOrigin &o) {
  if (T.yc < 0 || o.remY >= T.yt[T.ny - 1]) return T.TY;
  return o.remY * T.py;
}

// n / d with the planner's multiply-high constants (mul == 0: d == 1);
// exact for n < 2^31.
HPTT_HD inline int fast_div(int n, uint32_t mul, int shr) {
  return mul ? static_cast<int>(umulhi32(static_cast<uint32_t>(n), mul) >> shr) : n;
}

// Per-thread constants of a tile with one X dim, one Y dim and W == 1, from
// the thread index alone: load element x = tid % TX of rows q0 = tid / TX,
// store element y = tid % TY of columns qs0 = tid / TY; both slot maps are
// the identity, so shared memory holds (x, y) at y * LD + x.  Equal to the
// host table's entry (tile_thread_consts); the CPU replay checks that.
HPTT_HD inline HpttThr thread_consts_1d(const HpttProblem &P, const HpttTile &T, int tid) {
  HpttThr h;
  const int q0 = fast_div(tid, T.tx_mul, T.tx_shr);
  const int x = tid - q0 * T.TX;
  const int qs0 = fast_div(tid, T.ty_mul, T.ty_shr);
  const int y = tid - qs0 * T.TY;
  h.q0 = q0;
  h.qs0 = qs0;
  (void)P;
  h.inE = static_cast<int64_t>(x) * T.sxa;
  h.outE2 = static_cast<int64_t>(y) * T.syb;
  h.sme = x;
  h.sme2 = y * T.LD;
  h.cxe = T.xc >= 0 ? x : 0;
  h.cye2 = T.yc >= 0 ? y : 0;
  h.active = (tid < T.R1 * T.TX ? 1 : 0) | (tid < T.R2 * T.TY ? 2 : 0);
  h.pad = 0;
  return h;
}

// Walk of a thread's slots along a two-dim tile side (HpttWalk): slot q's
// first-dim digit and offset, then one step of R.  Unsigned offsets: the
// last step of a thread may pass the side's end (that slot is not
// accessed), and wraps instead of overflowing.
struct WalkPos {
  int d0;
  uint32_t off;
};

HPTT_HD inline WalkPos walk_start(const HpttWalk &w, int q) {
  const int d1 = fast_div(q, w.mul, w.shr);
  const int d0 = q - d1 * w.e0;
  WalkPos p;
  p.d0 = d0;
  p.off = static_cast<uint32_t>(d0) * static_cast<uint32_t>(w.s0) +
          static_cast<uint32_t>(d1) * static_cast<uint32_t>(w.s1);
  return p;
}

HPTT_HD inline void walk_step(const HpttWalk &w, WalkPos &p) {
  p.d0 += w.r0;
  p.off += static_cast<uint32_t>(w.step);
  if (p.d0 >= w.e0) {
    p.d0 -= w.e0;
    p.off += static_cast<uint32_t>(w.carry);
  }
}

// Iterations j >= 0 with q0 + j * R < lim (R > 0): ceil((lim - q0) / R), or 0.
HPTT_HD inline int valid_iters(int lim, int q0, uint32_t mul, int shr, int R) {
  return lim > q0 ? fast_div(lim - q0 + R - 1, mul, shr) : 0;
}


// Interior tile of an even single-dim shape (see tile_one): every loading
// thread has exactly J1 rows and every storing thread J2 columns.  Each phase
// runs with a compile-time trip count (N == J1 or J2, chosen by a chain of
// uniform compares once per phase): run-time bounds inside the unrolled loops
// compiled to a branch per access.  Offsets fit 32 bits (single-dim sides
// imply 32-bit tables, i.e. in-tile offsets below 2^31).
template <typename E, int N>
__device__ __forceinline__ void interior_load(const E *__restrict__ src, int stepA, E *s,
                                              int sstep) {
  E v[N];
#pragma unroll
  for (int j = 0; j < N; ++j) v[j] = __ldg(src + j * stepA);
#pragma unroll
  for (int j = 0; j < N; ++j) s[j * sstep] = v[j];
}

template <typename E, int MODE, bool UPD, int N>
__device__ __forceinline__ void interior_store(const E *s, int sstep, E *__restrict__ dst,
                                               int stepB, const Op<E, MODE, UPD> &op) {
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const E a = s[j * sstep];
    __stcs(dst + j * stepB, op(a, a));
  }
}

template <typename E, int N>
__device__ __forceinline__ void interior_load_n(int n, const E *__restrict__ src, int stepA,
                                                E *s, int sstep) {
  if (n == N) {
    interior_load<E, N>(src, stepA, s, sstep);
  } else if constexpr (N > 1) {
    interior_load_n<E, N - 1>(n, src, stepA, s, sstep);
  }
}

template <typename E, int MODE, bool UPD, int N>
__device__ __forceinline__ void interior_store_n(int n, const E *s, int sstep,
                                                 E *__restrict__ dst, int stepB,
                                                 const Op<E, MODE, UPD> &op) {
  if (n == N) {
    interior_store<E, MODE, UPD, N>(s, sstep, dst, stepB, op);
  } else if constexpr (N > 1) {
    interior_store_n<E, MODE, UPD, N - 1>(n, s, sstep, dst, stepB, op);
  }
}

template <typename E, int MODE, bool UPD>
__device__ __forceinline__ void tile_interior(const HpttTile &T, const E *__restrict__ A,
                                              E *__restrict__ B, const Op<E, MODE, UPD> &op,
                                              E *sdata, const HpttThr &th, const TileOrigin &o,
                                              int J1, int J2) {
  constexpr int J = hptt_jmax_tile(sizeof(E));
  const int sYf = static_cast<int>(T.sya);
  const int sXf = static_cast<int>(T.sxb);
  const int LD = T.LD, W = T.W, R1 = T.R1, R2 = T.R2;
  if (th.active & 1)
    interior_load_n<E, J>(J1, A + o.bA + th.inE + th.q0 * sYf, R1 * sYf,
                          sdata + th.q0 * LD + th.sme, R1 * LD);
  __syncthreads();
  if (th.active & 2)
    interior_store_n<E, MODE, UPD, J>(J2, sdata + th.sme2 + th.qs0 * W, R2 * W,
                                      B + o.bB + th.outE2 + th.qs0 * sXf, R2 * sXf, op);
}

// Edge or uneven tile of a single-dim copy/scale shape: the same compile-
// time loops as the interior, with every slot index clamped to the last
// valid row (column).  An iteration past the edge repeats that slot: it
// reads the same element again and writes the same value to the same place
// (a row slot in shared memory, a column of B), which changes nothing --
// so no per-element branch is needed.  Threads whose own element lies
// outside the tile skip their phase.
template <typename E, int N>
__device__ __forceinline__ void clamped_load(const E *__restrict__ src, int sY, int q0, int R1,
                                             int lim, E *s, int LD) {
  E v[N];
#pragma unroll
  for (int j = 0; j < N; ++j) v[j] = __ldg(src + min(q0 + j * R1, lim - 1) * sY);
#pragma unroll
  for (int j = 0; j < N; ++j) s[min(q0 + j * R1, lim - 1) * LD] = v[j];
}

template <typename E, int MODE, bool UPD, int N>
__device__ __forceinline__ void clamped_store(const E *s, int W, int qs0, int R2, int lim,
                                              E *__restrict__ dst, int sX,
                                              const Op<E, MODE, UPD> &op) {
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const int q = min(qs0 + j * R2, lim - 1);
    const E a = s[q * W];
    __stcs(dst + q * sX, op(a, a));
  }
}

template <typename E, int N>
__device__ __forceinline__ void clamped_load_n(int n, const E *__restrict__ src, int sY, int q0,
                                               int R1, int lim, E *s, int LD) {
  if (n == N) {
    clamped_load<E, N>(src, sY, q0, R1, lim, s, LD);
  } else if constexpr (N > 1) {
    clamped_load_n<E, N - 1>(n, src, sY, q0, R1, lim, s, LD);
  }
}

template <typename E, int MODE, bool UPD, int N>
__device__ __forceinline__ void clamped_store_n(int n, const E *s, int W, int qs0, int R2,
                                                int lim, E *__restrict__ dst, int sX,
                                                const Op<E, MODE, UPD> &op) {
  if (n == N) {
    clamped_store<E, MODE, UPD, N>(s, W, qs0, R2, lim, dst, sX, op);
  } else if constexpr (N > 1) {
    clamped_store_n<E, MODE, UPD, N - 1>(n, s, W, qs0, R2, lim, dst, sX, op);
  }
}

template <typename E, int MODE, bool UPD>
__device__ __forceinline__ void tile_clamped(const HpttTile &T, const E *__restrict__ A,
                                             E *__restrict__ B, const Op<E, MODE, UPD> &op,
                                             E *sdata, const HpttThr &th, const TileOrigin &o) {
  constexpr int J = hptt_jmax_tile(sizeof(E));
  const int TX = T.TX, TY = T.TY;
  const int limR = (T.yc >= 0 && o.remY < TY) ? o.remY : TY;
  const int limC = (T.xc >= 0 && o.remX < TX) ? o.remX : TX;
  if ((th.active & 1) && th.cxe < o.remX)
    clamped_load_n<E, J>(T.J1, A + o.bA + th.inE, static_cast<int>(T.sya), th.q0, T.R1, limR,
                         sdata + th.sme, T.LD);
  __syncthreads();
  if ((th.active & 2) && th.cye2 < o.remY)
    clamped_store_n<E, MODE, UPD, J>(T.J2, sdata + th.sme2, T.W, th.qs0, T.R2, limC,
                                     B + o.bB + th.outE2, static_cast<int>(T.sxb), op);
}

// Single-dim tiles that also read B, shapes with J1 == J2 == J: one
// compile-time instance (the B values must live across the barrier, so the
// two phases cannot be dispatched separately).
// Interior tile of an even shape: no bounds at all.
template <typename E, int MODE, bool UPD>
__device__ __forceinline__ void tile_interior_upd(const HpttTile &T, const E *__restrict__ A,
                                                  E *__restrict__ B, const Op<E, MODE, UPD> &op,
                                                  E *sdata, const HpttThr &th,
                                                  const TileOrigin &o) {
  constexpr int J = hptt_jmax_tile(sizeof(E));
  const int sYf = static_cast<int>(T.sya);
  const int sXf = static_cast<int>(T.sxb);
  const int LD = T.LD, W = T.W, R1 = T.R1, R2 = T.R2;
  const bool ld = th.active & 1, st = th.active & 2;
  const E *src = A + o.bA + th.inE + th.q0 * sYf;
  E *dst = B + o.bB + th.outE2 + th.qs0 * sXf;
  const int stepA = R1 * sYf, stepB = R2 * sXf;
  E v[J], bv[J];
  if (ld) {
#pragma unroll
    for (int j = 0; j < J; ++j) v[j] = __ldg(src + j * stepA);
  }
  if (st) {
#pragma unroll
    for (int j = 0; j < J; ++j) bv[j] = dst[j * stepB];
  }
  if (ld) {
    E *s = sdata + th.q0 * LD + th.sme;
#pragma unroll
    for (int j = 0; j < J; ++j) s[j * R1 * LD] = v[j];
  }
  __syncthreads();
  if (st) {
    const E *s = sdata + th.sme2 + th.qs0 * W;
#pragma unroll
    for (int j = 0; j < J; ++j) dst[j * stepB] = op(s[j * R2 * W], bv[j]);
  }
}

// Edge tile: slot indices clamped as in tile_clamped; every B value is read
// before the barrier, so a repeated column computes and writes the same
// value again.  (Used for 8- and 16-byte elements: with 4-byte elements' 16
// iterations it needs too many registers, and their edge tiles take the
// general path.)
template <typename E, int MODE, bool UPD>
__device__ __forceinline__ void tile_full_upd(const HpttTile &T, const E *__restrict__ A,
                                              E *__restrict__ B, const Op<E, MODE, UPD> &op,
                                              E *sdata, const HpttThr &th,
                                              const TileOrigin &o) {
  constexpr int J = hptt_jmax_tile(sizeof(E));
  const int sY = static_cast<int>(T.sya);
  const int sX = static_cast<int>(T.sxb);
  const int LD = T.LD, W = T.W, R1 = T.R1, R2 = T.R2;
  const int limR = T.yc >= 0 && o.remY < T.TY ? o.remY : T.TY;
  const int limC = T.xc >= 0 && o.remX < T.TX ? o.remX : T.TX;
  const bool ld = (th.active & 1) && th.cxe < o.remX;
  const bool st = (th.active & 2) && th.cye2 < o.remY;
  const E *src = A + o.bA + th.inE;
  E *dst = B + o.bB + th.outE2;
  E v[J], bv[J];
  if (ld) {
#pragma unroll
    for (int j = 0; j < J; ++j) v[j] = __ldg(src + min(th.q0 + j * R1, limR - 1) * sY);
  }
  if (st) {
#pragma unroll
    for (int j = 0; j < J; ++j) bv[j] = dst[min(th.qs0 + j * R2, limC - 1) * sX];
  }
  if (ld) {
#pragma unroll
    for (int j = 0; j < J; ++j) sdata[min(th.q0 + j * R1, limR - 1) * LD + th.sme] = v[j];
  }
  __syncthreads();
  if (st) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int q = min(th.qs0 + j * R2, limC - 1);
      dst[q * sX] = op(sdata[th.sme2 + q * W], bv[j]);
    }
  }
}

// Run f with a compile-time trip count equal to n (1 <= n <= N): a chain of
// uniform compares, once per phase.
template <int N>
struct TripCount {
  static constexpr int value = N;
};

template <int N, typename F>
__device__ __forceinline__ void with_trip_count(int n, F &&f) {
  if (n == N) {
    f(TripCount<N>());
  } else if constexpr (N > 1) {
    with_trip_count<N - 1>(n, f);
  }
}

// How a tile side yields the offsets of a thread's slots q0 + j * R:
// q * stride (one dim), a walk (two dims, HpttWalk) or the side's table.
enum SideKind : int { SIDE_AFFINE = 0, SIDE_WALK = 1, SIDE_TABLE = 2 };

template <int KIND, typename OffT>
struct SideSlots {
  int q;        // current slot
  WalkPos w;    // SIDE_WALK
  __device__ __forceinline__ SideSlots(int q0, const HpttWalk &wk) : q(q0) {
    if (KIND == SIDE_WALK) w = walk_start(wk, q0);
  }
  // offset of the current slot; `ok`: the slot is inside the side
  __device__ __forceinline__ OffT offset(bool ok, int stride,
                                         const HpttTabEnt<OffT> *__restrict__ tab) const {
    if (KIND == SIDE_AFFINE) return static_cast<OffT>(q * stride);
    if (KIND == SIDE_WALK) return static_cast<OffT>(w.off);
    return tab[ok ? q : 0].off;
  }
  __device__ __forceinline__ void next(int R, const HpttWalk &wk) {
    q += R;
    if (KIND == SIDE_WALK) walk_step(wk, w);
  }
};

// Interior tile of a table-driven shape (a side with several dims, or the
// 64-bit-offset kernel): every chunk coordinate is inside the tensor, so no
// offset needs a check.  Compile-time trip counts per phase (N = J1 or J2);
// a thread's slot q0 + j*R (q0 < R) can pass the side's end only at its
// last iteration, which alone is tested.  Every slot is loaded, read and
// written by exactly one thread.  Update tiles read their B values before
// the barrier.
template <typename E, int MODE, bool UPD, typename OffT, int XK, int YK>
__device__ __forceinline__ void tile_table_interior_k(
    const HpttTile &T, const E *__restrict__ A, E *__restrict__ B,
    const HpttTabEnt<OffT> *__restrict__ tabY, const HpttTabEnt<OffT> *__restrict__ tabX,
    const Op<E, MODE, UPD> &op, E *sdata, const HpttThr &th, const TileOrigin &o) {
  constexpr int J = hptt_jmax_tile(sizeof(E));
  const int LD = T.LD, W = T.W, R1 = T.R1, R2 = T.R2, TX = T.TX, TY = T.TY;
  const int sY = YK == SIDE_AFFINE ? static_cast<int>(T.sya) : 0;
  const int sX = XK == SIDE_AFFINE ? static_cast<int>(T.sxb) : 0;
  const E *src = A + o.bA + th.inE;
  E *dst = B + o.bB + th.outE2;
  const bool ld = th.active & 1, st = th.active & 2;
  E bv[UPD ? J : 1];
  if (UPD && st) {
    with_trip_count<J>(T.J2, [&](auto n) {
      constexpr int N = decltype(n)::value;
      SideSlots<XK, OffT> x(th.qs0, T.wx);
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const bool ok = j < N - 1 || x.q < TX;
        const OffT off = x.offset(ok, sX, tabX);
        if (ok) bv[UPD ? j : 0] = dst[off];
        x.next(R2, T.wx);
      }
    });
  }
  if (ld) {
    with_trip_count<J>(T.J1, [&](auto n) {
      constexpr int N = decltype(n)::value;
      SideSlots<YK, OffT> y(th.q0, T.wy);
      E v[N];
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const bool ok = j < N - 1 || y.q < TY;
        const OffT off = y.offset(ok, sY, tabY);
        if (ok) v[j] = __ldg(src + off);
        y.next(R1, T.wy);
      }
      E *s = sdata + th.sme + th.q0 * LD;
#pragma unroll
      for (int j = 0; j < N; ++j)
        if (j < N - 1 || th.q0 + j * R1 < TY) s[j * R1 * LD] = v[j];
    });
  }
  __syncthreads();
  if (st) {
    with_trip_count<J>(T.J2, [&](auto n) {
      constexpr int N = decltype(n)::value;
      SideSlots<XK, OffT> x(th.qs0, T.wx);
      const E *s = sdata + th.sme2 + th.qs0 * W;
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const bool ok = j < N - 1 || x.q < TX;
        const OffT off = x.offset(ok, sX, tabX);
        if (ok) {
          const E a = s[j * R2 * W];
          if (UPD)
            dst[off] = op(a, bv[UPD ? j : 0]);
          else
            __stcs(dst + off, op(a, a));
        }
        x.next(R2, T.wx);
      }
    });
  }
}

// The same tile for kernels that keep persistent-loop state (fewer live
// registers): every phase runs all N iterations with slots past the side's
// end clamped to the last one, which repeats it (same element, same value);
// copy and scale tiles only.
template <typename E, int MODE, bool UPD, typename OffT, bool LX, bool LY>
__device__ __forceinline__ void tile_table_interior_clamped(
    const HpttTile &T, const E *__restrict__ A, E *__restrict__ B,
    const HpttTabEnt<OffT> *__restrict__ tabY, const HpttTabEnt<OffT> *__restrict__ tabX,
    const Op<E, MODE, UPD> &op, E *sdata, const HpttThr &th, const TileOrigin &o) {
  constexpr int J = hptt_jmax_tile(sizeof(E));
  const int LD = T.LD, W = T.W, R1 = T.R1, R2 = T.R2, TX = T.TX, TY = T.TY;
  const int sY = LY ? static_cast<int>(T.sya) : 0;
  const int sX = LX ? static_cast<int>(T.sxb) : 0;
  if (th.active & 1) {
    const E *src = A + o.bA + th.inE;
    with_trip_count<J>(T.J1, [&](auto n) {
      constexpr int N = decltype(n)::value;
      E v[N];
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const int q = min(th.q0 + j * R1, TY - 1);
        v[j] = __ldg(src + (LY ? static_cast<OffT>(q * sY) : tabY[q].off));
      }
      E *s = sdata + th.sme;
#pragma unroll
      for (int j = 0; j < N; ++j) s[min(th.q0 + j * R1, TY - 1) * LD] = v[j];
    });
  }
  __syncthreads();
  if (th.active & 2) {
    E *dst = B + o.bB + th.outE2;
    with_trip_count<J>(T.J2, [&](auto n) {
      constexpr int N = decltype(n)::value;
      const E *s = sdata + th.sme2;
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const int q = min(th.qs0 + j * R2, TX - 1);
        const E a = s[q * W];
        __stcs(dst + (LX ? static_cast<OffT>(q * sX) : tabX[q].off), op(a, a));
      }
    });
  }
}

// Side kinds of a table-driven interior tile, chosen once per tile (uniform);
// without WALK every multi-dim side reads its table.
template <typename E, int MODE, bool UPD, typename OffT, bool LX, bool LY, bool WALK>
__device__ __forceinline__ void tile_table_interior(const HpttTile &T, const E *__restrict__ A,
                                                    E *__restrict__ B,
                                                    const HpttTabEnt<OffT> *__restrict__ tabY,
                                                    const HpttTabEnt<OffT> *__restrict__ tabX,
                                                    const Op<E, MODE, UPD> &op, E *sdata,
                                                    const HpttThr &th, const TileOrigin &o) {
  if constexpr (!WALK) {
    tile_table_interior_clamped<E, MODE, UPD, OffT, LX, LY>(T, A, B, tabY, tabX, op, sdata, th,
                                                            o);
  } else if constexpr (sizeof(OffT) > 4) {
    tile_table_interior_k<E, MODE, UPD, OffT, SIDE_TABLE, SIDE_TABLE>(T, A, B, tabY, tabX, op,
                                                                      sdata, th, o);
  } else if constexpr (!WALK) {
    tile_table_interior_clamped<E, MODE, UPD, OffT, LX, LY>(T, A, B, tabY, tabX, op, sdata, th,
                                                            o);
  } else {
    constexpr int XA = LX ? SIDE_AFFINE : SIDE_WALK;
    constexpr int YA = LY ? SIDE_AFFINE : SIDE_WALK;
    const bool xt = !LX && T.wx.e0 == 0, yt = !LY && T.wy.e0 == 0;
    if (!xt && !yt)
      tile_table_interior_k<E, MODE, UPD, OffT, XA, YA>(T, A, B, tabY, tabX, op, sdata, th, o);
    else if (!xt)
      tile_table_interior_k<E, MODE, UPD, OffT, XA, SIDE_TABLE>(T, A, B, tabY, tabX, op, sdata,
                                                                th, o);
    else if (!yt)
      tile_table_interior_k<E, MODE, UPD, OffT, SIDE_TABLE, YA>(T, A, B, tabY, tabX, op, sdata,
                                                                th, o);
    else
      tile_table_interior_k<E, MODE, UPD, OffT, SIDE_TABLE, SIDE_TABLE>(T, A, B, tabY, tabX, op,
                                                                        sdata, th, o);
  }
}

// ---------------------------------------------------------------------------
// One tile through shared memory (one CTA).
//
// Shared memory holds element (w, x, y) at row qrow(y), column
// qcol(x) * W + w, where qrow enumerates the Y dims in INPUT order and qcol
// the X dims in OUTPUT order; the host folds both permutations into the
// per-thread constants, so neither phase indexes through a table.
// Load phase: thread (e, q0) reads rows q = q0 + j*R1 of its element e --
// input-contiguous runs -- plus, when B is read, the B elements it combines
// later.  Store phase: thread (e2, qs0) writes columns q = qs0 + j*R2 of its
// element e2 -- output-contiguous runs.
//
// LX / LY: the X (Y) side has at most one dim, so slot q IS that dim's
// coordinate: offset q * stride and validity q < remaining extent, with no
// table read (the tables hold exactly these values; the CPU replay checks
// that).
// ---------------------------------------------------------------------------
// FAST: the forms that need more registers -- update tiles' bounds-free and
// clamped forms, walked two-dim sides -- are allowed (kernels that also keep
// persistent-loop state turn it off).
template <typename E, int MODE, bool UPD, typename OffT, bool LX, bool LY, bool FAST = true>
__device__ __forceinline__ void tile_one(const HpttProblem &P, const HpttTile &T,
                                         const E *__restrict__ A, E *__restrict__ B,
                                         const unsigned char *__restrict__ tables,
                                         const Op<E, MODE, UPD> &op, E *sdata, uint32_t tile) {
  constexpr int J = hptt_jmax_tile(sizeof(E));
  using Ent = HpttTabEnt<OffT>;
  const Ent *__restrict__ tabY = reinterpret_cast<const Ent *>(tables);
  const Ent *__restrict__ tabX = reinterpret_cast<const Ent *>(tables + T.tab2_off);
  // single-dim sides with W == 1: constants from the thread index (no table
  // read before the first load); else the host table's entry
  const HpttThr th = (LX && LY && T.W == 1 && T.nx == 1 && T.ny == 1)
                         ? thread_consts_1d(P, T, threadIdx.x)
                         : reinterpret_cast<const HpttThr *>(tables + T.thr_off)[threadIdx.x];
  const TileOrigin o = tile_origin(P, T, tile);
  const int LD = T.LD, W = T.W, R1 = T.R1, R2 = T.R2, J1 = T.J1, J2 = T.J2;
  const int TX = T.TX, TY = T.TY;
  // Iteration j of a thread covers slot q0 + j*R1 (q0 < R1), so the slot
  // bound q < TY already implies j < J1: the loops test only the slot bound.
  if (UPD && FAST && LX && LY && J1 == J && J2 == J) {
    // (the clamped edge form needs too many registers with 4-byte
    // elements' 16 iterations; their edge tiles take the general path)
    if (T.even && o.remX >= TX && o.remY >= TY) {
      tile_interior_upd<E, MODE, UPD>(T, A, B, op, sdata, th, o);
      return;
    }
    if constexpr (sizeof(E) > 4) {
      tile_full_upd<E, MODE, UPD>(T, A, B, op, sdata, th, o);
      return;
    }
  }
  if (!UPD && LX && LY && T.even && o.remX >= TX && o.remY >= TY) {
    // Interior tile of an even shape: every loading thread has exactly J1
    // rows and every storing thread J2 columns (TY == R1*J1, TX == R2*J2),
    // so the accesses -- the same as the general path's -- need no
    // per-element bounds.
    tile_interior<E, MODE, UPD>(T, A, B, op, sdata, th, o, J1, J2);
    return;
  }
  if (!UPD && LX && LY) {
    tile_clamped<E, MODE, UPD>(T, A, B, op, sdata, th, o);
    return;
  }
  if constexpr (!UPD || FAST) {
    // interior tiles with a multi-dim side, and update tiles with single-dim
    // sides that the forms above did not take
    if ((!(LX && LY) || (UPD && T.upd_exact)) && o.remX >= T.xce && o.remY >= T.yce) {
      tile_table_interior<E, MODE, UPD, OffT, LX, LY, FAST>(T, A, B, tabY, tabX, op, sdata, th,
                                                            o);
      return;
    }
  }
  const bool ld_ok = (th.active & 1) && th.cxe < o.remX;
  const bool st_ok = (th.active & 2) && th.cye2 < o.remY;
  const int sY = LY ? static_cast<int>(T.sya) : 0;
  const int sX = LX ? static_cast<int>(T.sxb) : 0;
  const int limQY = (LY && T.yc >= 0 && o.remY < TY) ? o.remY : TY;
  const int limQX = (LX && T.xc >= 0 && o.remX < TX) ? o.remX : TX;
  E v[J];
  if (ld_ok) {
    const E *src = A + o.bA + th.inE;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int q = th.q0 + j * R1;
      if (LY) {
        if (q < limQY) v[j] = __ldg(src + q * sY);
      } else if (q < TY) {
        const Ent en = tabY[q];
        v[j] = __ldg(src + (en.c < o.remY ? en.off : OffT(0)));
      }
    }
  }
  E *dst = B + o.bB + th.outE2;
  E bv[J];
  if (UPD && st_ok) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int q = th.qs0 + j * R2;
      if (LX) {
        if (q < limQX) bv[j] = dst[q * sX];
      } else if (q < TX) {
        const Ent en = tabX[q];
        bv[j] = dst[en.c < o.remX ? en.off : OffT(0)];
      }
    }
  }
  if (ld_ok) {
    E *s = sdata + th.q0 * LD + th.sme;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int q = th.q0 + j * R1;
      if (q < (LY ? limQY : TY)) s[j * R1 * LD] = v[j];
    }
  }
  __syncthreads();
  if (!st_ok) return;
  const E *s = sdata + th.sme2 + th.qs0 * W;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int q = th.qs0 + j * R2;
    bool ok;
    int64_t off;
    if (LX) {
      ok = q < limQX;
      off = q * sX;
    } else {
      ok = q < TX;
      Ent en{};
      if (ok) en = tabX[q];
      ok = ok && en.c < o.remX;
      off = static_cast<int64_t>(en.off);
    }
    if (ok) {
      const E a = s[j * R2 * W];
      const E r = op(a, UPD ? bv[j] : a);
      if (UPD) dst[off] = r; else __stcs(dst + off, r);
    }
  }
}

// ---------------------------------------------------------------------------
// One tile of rows (shared stride-1 dim); VEC elements per access.  Dim 0
// has stride 1 in A and B whenever VEC > 1 (checked by the planner).
// ---------------------------------------------------------------------------
template <typename E, int MODE, bool UPD, typename OffT, int VEC>
__device__ __forceinline__ void rows_one(const HpttProblem &P, const HpttTile &T,
                                         const E *__restrict__ A, E *__restrict__ B,
                                         const unsigned char *__restrict__ tables,
                                         const Op<E, MODE, UPD> &op, uint32_t tile) {
  constexpr int J = hptt_jmax_rows(sizeof(E) * VEC);
  const RowThread s = rows_thread(T, threadIdx.x);
  if (!s.active) return;
  const TileOrigin o = tile_origin(P, T, tile);
  const int64_t col = static_cast<int64_t>(s.e) * VEC;
  if (col >= o.remX) return;
  const int n = min(T.J1, valid_iters(rows_limit_y(T, o), s.y0, T.r1_mul, T.r1_shr, T.R1));
  const OffT *__restrict__ tabA = reinterpret_cast<const OffT *>(tables);
  const OffT *__restrict__ tabB = reinterpret_cast<const OffT *>(tables + T.tab2_off);
  const E *src = A + o.bA + col * P.sA[0];
  E *dst = B + o.bB + col * P.sB[0];
  const int R1 = T.R1;
  if (rows_limit_y(T, o) == T.TY) {
    // Interior tile: compile-time trip count J1; a thread's row y0 + j*R1
    // (y0 < R1) can pass TY only at its last iteration.  Row offsets come
    // from the tables even for one Y dim: a warp's lanes read the same entry
    // (one broadcast), which measured faster than 64-bit y * stride.
    const int y0 = s.y0, TY = T.TY;
    with_trip_count<J>(T.J1, [&](auto nn) {
      constexpr int N = decltype(nn)::value;
      Vec<E, VEC> av[N];
      Vec<E, VEC> bv[UPD ? N : 1];
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const int y = y0 + j * R1;
        if (j < N - 1 || y < TY) {
          av[j] = ld_vec<E, VEC>(src + __ldg(tabA + y));
          if (UPD) bv[UPD ? j : 0] = ld_vec_rw<E, VEC>(dst + __ldg(tabB + y));
        }
      }
#pragma unroll
      for (int j = 0; j < N; ++j) {
        const int y = y0 + j * R1;
        if (j < N - 1 || y < TY) {
          Vec<E, VEC> r;
#pragma unroll
          for (int k = 0; k < VEC; ++k)
            r.v[k] = op(av[j].v[k], UPD ? bv[UPD ? j : 0].v[k] : av[j].v[k]);
          st_vec<E, VEC>(dst + __ldg(tabB + y), r);
        }
      }
    });
    return;
  }
  Vec<E, VEC> av[J];
  Vec<E, VEC> bv[J];
#pragma unroll
  for (int j = 0; j < J; ++j) {
    if (j < n) {
      const int y = s.y0 + j * R1;
      av[j] = ld_vec<E, VEC>(src + __ldg(tabA + y));
      if (UPD) bv[j] = ld_vec_rw<E, VEC>(dst + __ldg(tabB + y));
    }
  }
#pragma unroll
  for (int j = 0; j < J; ++j) {
    if (j < n) {
      const int y = s.y0 + j * R1;
      Vec<E, VEC> r;
#pragma unroll
      for (int k = 0; k < VEC; ++k) r.v[k] = op(av[j].v[k], UPD ? bv[j].v[k] : av[j].v[k]);
      st_vec<E, VEC>(dst + __ldg(tabB + y), r);
    }
  }
}

}  // namespace dev
}  // namespace hptt_b200
