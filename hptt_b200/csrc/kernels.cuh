// sm_100a device code for B = alpha * A(perm) + beta * B.
//
// Replaces the reference's CPU macro/micro kernels
// (src/kernels/macro_kernel_trans.cc, src/arch/avx2/kernel_trans_avx2.cc):
//   tile_body  -- the in-register W x W transposes (kernel_trans_avx2.cc:21-467)
//                 become a shared-memory tile that pairs the input's stride-1
//                 dims with the output's, read and written in contiguous runs;
//                 ragged edges (the reference's scalar kernels,
//                 macro_kernel_trans.cc:225-252) are predicated in the same
//                 pass.
//   rows_body  -- the shared-stride-1 linear kernel (kernel_trans_avx2.cc:480-530,
//                 macro_kernel_trans.cc:181-195) becomes a vectorised copy-scale
//                 over rows.
// Both fuse the beta * B read into the same pass and are written so one CTA
// can also run them on tiles of many different problems (batched form).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "desc.h"

namespace hptt_b200 {
namespace dev {


// ---------------------------------------------------------------------------
// Element arithmetic.  Products and sums are rounded separately (no FMA), in
// the reference's order (src/arch/avx2/kernel_trans_avx2.cc:68-107).
// ---------------------------------------------------------------------------
struct Scal {
  double ar, ai, br, bi;
};

template <typename E, int MODE, bool UPD>
struct Op;

// bit copy (alpha == 1, B not read)
template <typename E>
struct Op<E, MODE_COPY, false> {
  __device__ __forceinline__ explicit Op(const Scal &) {}
  __device__ __forceinline__ E operator()(E a, E) const { return a; }
};

template <bool UPD>
struct Op<float, MODE_REAL, UPD> {
  float al, be;
  __device__ __forceinline__ explicit Op(const Scal &s)
      : al(static_cast<float>(s.ar)), be(static_cast<float>(s.br)) {}
  __device__ __forceinline__ float operator()(float a, float b) const {
    float t = __fmul_rn(al, a);
    if (UPD) t = __fadd_rn(t, __fmul_rn(be, b));
    return t;
  }
};

template <bool UPD>
struct Op<double, MODE_REAL, UPD> {
  double al, be;
  __device__ __forceinline__ explicit Op(const Scal &s) : al(s.ar), be(s.br) {}
  __device__ __forceinline__ double operator()(double a, double b) const {
    double t = __dmul_rn(al, a);
    if (UPD) t = __dadd_rn(t, __dmul_rn(be, b));
    return t;
  }
};

template <bool UPD>
struct Op<float2, MODE_REAL, UPD> {
  float al, be;
  __device__ __forceinline__ explicit Op(const Scal &s)
      : al(static_cast<float>(s.ar)), be(static_cast<float>(s.br)) {}
  __device__ __forceinline__ float2 operator()(float2 a, float2 b) const {
    float2 t;
    t.x = __fmul_rn(al, a.x);
    t.y = __fmul_rn(al, a.y);
    if (UPD) {
      t.x = __fadd_rn(t.x, __fmul_rn(be, b.x));
      t.y = __fadd_rn(t.y, __fmul_rn(be, b.y));
    }
    return t;
  }
};

template <bool UPD>
struct Op<double2, MODE_REAL, UPD> {
  double al, be;
  __device__ __forceinline__ explicit Op(const Scal &s) : al(s.ar), be(s.br) {}
  __device__ __forceinline__ double2 operator()(double2 a, double2 b) const {
    double2 t;
    t.x = __dmul_rn(al, a.x);
    t.y = __dmul_rn(al, a.y);
    if (UPD) {
      t.x = __dadd_rn(t.x, __dmul_rn(be, b.x));
      t.y = __dadd_rn(t.y, __dmul_rn(be, b.y));
    }
    return t;
  }
};

// complex scalars: re = fl(fl(sr*xr) - fl(si*xi)), im = fl(fl(sr*xi) + fl(si*xr))
template <bool UPD>
struct Op<float2, MODE_CPLX, UPD> {
  float ar, ai, br, bi;
  __device__ __forceinline__ explicit Op(const Scal &s)
      : ar(static_cast<float>(s.ar)), ai(static_cast<float>(s.ai)),
        br(static_cast<float>(s.br)), bi(static_cast<float>(s.bi)) {}
  __device__ __forceinline__ float2 operator()(float2 a, float2 b) const {
    float2 t;
    t.x = __fsub_rn(__fmul_rn(ar, a.x), __fmul_rn(ai, a.y));
    t.y = __fadd_rn(__fmul_rn(ar, a.y), __fmul_rn(ai, a.x));
    if (UPD) {
      const float ux = __fsub_rn(__fmul_rn(br, b.x), __fmul_rn(bi, b.y));
      const float uy = __fadd_rn(__fmul_rn(br, b.y), __fmul_rn(bi, b.x));
      t.x = __fadd_rn(t.x, ux);
      t.y = __fadd_rn(t.y, uy);
    }
    return t;
  }
};

template <bool UPD>
struct Op<double2, MODE_CPLX, UPD> {
  double ar, ai, br, bi;
  __device__ __forceinline__ explicit Op(const Scal &s)
      : ar(s.ar), ai(s.ai), br(s.br), bi(s.bi) {}
  __device__ __forceinline__ double2 operator()(double2 a, double2 b) const {
    double2 t;
    t.x = __dsub_rn(__dmul_rn(ar, a.x), __dmul_rn(ai, a.y));
    t.y = __dadd_rn(__dmul_rn(ar, a.y), __dmul_rn(ai, a.x));
    if (UPD) {
      const double ux = __dsub_rn(__dmul_rn(br, b.x), __dmul_rn(bi, b.y));
      const double uy = __dadd_rn(__dmul_rn(br, b.y), __dmul_rn(bi, b.x));
      t.x = __dadd_rn(t.x, ux);
      t.y = __dadd_rn(t.y, uy);
    }
    return t;
  }
};

// ---------------------------------------------------------------------------
// Memory helpers
// ---------------------------------------------------------------------------
template <typename E>
__device__ __forceinline__ E ld_in(const E *p) { return __ldg(p); }

template <typename E>
__device__ __forceinline__ void st_out(E *p, E v, bool stream) {
  if (stream) __stcs(p, v); else *p = v;
}

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
__device__ __forceinline__ void st_vec(E *p, const Vec<E, VEC> &v, bool stream) {
  using R = typename RawT<sizeof(E) * VEC>::T;
  R r;
  memcpy(&r, &v, sizeof(r));
  if (stream) __stcs(reinterpret_cast<R *>(p), r);
  else *reinterpret_cast<R *>(p) = r;
}

// ---------------------------------------------------------------------------
// Tile geometry shared by every tile of one problem.
// ---------------------------------------------------------------------------
struct TileOrigin {
  int64_t bA, bB;   // element offsets of the tile origin in A and B
  int64_t remX;     // extent left along the chunked X dim (or W dim), or big
  int64_t remY;     // extent left along the chunked Y dim, or big
  bool interior;    // every element of the tile is inside the tensor
};

HPTT_HD inline TileOrigin tile_origin(const HpttProblem &P, const HpttTile &T,
                                      uint32_t tile) {
  TileOrigin o;
  o.bA = 0;
  o.bB = 0;
  o.remX = INT64_MAX;
  o.remY = INT64_MAX;
  uint32_t rem = tile;
  const int xc = (T.kind == KIND_ROWS) ? T.wc : T.xc;
  for (int g = 0; g < T.ng; ++g) {
    const uint32_t cnt = T.gcnt[g];
    const uint32_t c = rem % cnt;
    rem /= cnt;
    const int d = T.gd[g];
    const int64_t pos = static_cast<int64_t>(c) * T.gstep[g];
    o.bA += pos * P.sA[d];
    o.bB += pos * P.sB[d];
    if (d == xc) o.remX = P.n[d] - pos;
    if (d == T.yc) o.remY = P.n[d] - pos;
  }
  int64_t xt = 1, yt = 1;
  if (T.kind == KIND_ROWS) {
    xt = T.W;
  } else if (T.nx) {
    xt = T.xt[T.nx - 1];
  }
  if (T.ny) yt = T.yt[T.ny - 1];
  o.interior = o.remX >= xt && o.remY >= yt;
  return o;
}

// Mixed-radix decomposition of a tile-local index over a list of dims.
template <typename OffT>
HPTT_HD inline void decompose(int idx, int nd, const int32_t *dims, const int32_t *ext,
                              const int64_t *stride, int chunk_dim, OffT *off,
                              int *chunk_c) {
  OffT o = 0;
  int cc = 0;
  for (int i = 0; i < nd; ++i) {
    const int c = idx % ext[i];
    idx /= ext[i];
    o += static_cast<OffT>(c) * static_cast<OffT>(stride[dims[i]]);
    if (dims[i] == chunk_dim) cc = c;
  }
  *off = o;
  *chunk_c = cc;
}

// Per-thread state of the shared-memory tile transpose.
template <typename OffT>
struct TileThread {
  bool ld_active, st_active;
  int y0, x0;
  OffT inE, outE2;
  int cxe, cye2;
  int sme, sme2;
};

// Fill the y/x tables (shared memory on the device): threads tid,
// tid + nthreads, ... each fill one entry.  Callers __syncthreads() after.
template <typename OffT>
HPTT_HD inline void tile_tables(const HpttProblem &P, const HpttTile &T, OffT *tInY,
                                int *tCy, OffT *tOutX, int *tCx, int tid, int nthreads) {
  for (int y = tid; y < T.TY; y += nthreads) {
    OffT o;
    int c;
    decompose<OffT>(y, T.ny, T.yd, T.yt, P.sA, T.yc, &o, &c);
    tInY[y] = o;
    tCy[y] = c;
  }
  for (int x = tid; x < T.TX; x += nthreads) {
    OffT o;
    int c;
    decompose<OffT>(x, T.nx, T.xd, T.xt, P.sB, T.xc, &o, &c);
    tOutX[x] = o;
    tCx[x] = c;
  }
}

// Per-thread constants of the tile transpose (independent of the tile).
template <typename OffT>
HPTT_HD inline TileThread<OffT> tile_thread(const HpttProblem &P, const HpttTile &T,
                                            int tid) {
  TileThread<OffT> s;
  s.ld_active = tid < T.R1 * T.RW;
  {
    const int e = tid % T.RW;
    const int w = e % T.W, x = e / T.W;
    OffT o;
    int c;
    decompose<OffT>(x, T.nx, T.xd, T.xt, P.sA, T.xc, &o, &c);
    s.inE = o + static_cast<OffT>(w) * static_cast<OffT>(P.sA[0]);
    s.cxe = c;
    s.y0 = tid / T.RW;
    s.sme = e;
  }
  s.st_active = tid < T.R2 * T.WTY;
  {
    const int e2 = tid % T.WTY;
    const int w = e2 % T.W, y = e2 / T.W;
    OffT o;
    int c;
    decompose<OffT>(y, T.ny, T.yd, T.yt, P.sB, T.yc, &o, &c);
    s.outE2 = o + static_cast<OffT>(w) * static_cast<OffT>(P.sB[0]);
    s.cye2 = c;
    s.x0 = tid / T.WTY;
    s.sme2 = y * T.LD + w;
  }
  return s;
}

// One tile through shared memory.  sdata holds TY rows of LD elements.
template <typename E, int MODE, bool UPD, typename OffT>
__device__ __forceinline__ void tile_body(const HpttTile &T, const E *__restrict__ A,
                                          E *__restrict__ B, const Op<E, MODE, UPD> &op,
                                          const TileThread<OffT> &s, const TileOrigin &o,
                                          E *sdata, const OffT *tInY, const int *tCy,
                                          const OffT *tOutX, const int *tCx) {
  constexpr int kJMax = hptt_jmax_tile(sizeof(E));
  // load phase: rows y, element e (input-contiguous)
  if (s.ld_active) {
    E v[kJMax];
    const E *src = A + o.bA + s.inE;
#pragma unroll
    for (int j = 0; j < kJMax; ++j) {
      const int y = s.y0 + j * T.R1;
      if (j < T.J1 && y < T.TY) {
        if (o.interior || (s.cxe < o.remX && tCy[y] < o.remY)) v[j] = ld_in(src + tInY[y]);
      }
    }
#pragma unroll
    for (int j = 0; j < kJMax; ++j) {
      const int y = s.y0 + j * T.R1;
      if (j < T.J1 && y < T.TY) sdata[y * T.LD + s.sme] = v[j];
    }
  }
  __syncthreads();
  // store phase: columns x, element e2 (output-contiguous)
  if (s.st_active) {
    E *dst = B + o.bB + s.outE2;
    E bv[kJMax];
    if (UPD) {
#pragma unroll
      for (int j = 0; j < kJMax; ++j) {
        const int x = s.x0 + j * T.R2;
        if (j < T.J2 && x < T.TX) {
          if (o.interior || (s.cye2 < o.remY && tCx[x] < o.remX)) bv[j] = dst[tOutX[x]];
        }
      }
    }
#pragma unroll
    for (int j = 0; j < kJMax; ++j) {
      const int x = s.x0 + j * T.R2;
      if (j < T.J2 && x < T.TX) {
        if (o.interior || (s.cye2 < o.remY && tCx[x] < o.remX)) {
          const E a = sdata[s.sme2 + x * T.W];
          st_out(dst + tOutX[x], op(a, bv[j]), !UPD);
        }
      }
    }
  }
  __syncthreads();
}

// Per-thread state of the row copy.
template <typename OffT>
struct RowThread {
  bool active;
  int e;   // vector index inside the row chunk
  int y0;
};

template <typename OffT>
HPTT_HD inline void rows_tables(const HpttProblem &P, const HpttTile &T, OffT *tInY,
                                OffT *tOutY, int *tCy, int tid, int nthreads) {
  for (int y = tid; y < T.TY; y += nthreads) {
    OffT oa, ob;
    int c;
    decompose<OffT>(y, T.ny, T.yd, T.yt, P.sA, T.yc, &oa, &c);
    decompose<OffT>(y, T.ny, T.yd, T.yt, P.sB, T.yc, &ob, &c);
    tInY[y] = oa;
    tOutY[y] = ob;
    tCy[y] = c;
  }
}

template <typename OffT>
HPTT_HD inline RowThread<OffT> rows_thread(const HpttTile &T, int tid) {
  RowThread<OffT> s;
  s.active = tid < T.R1 * T.RW;
  s.e = tid % T.RW;
  s.y0 = tid / T.RW;
  return s;
}

// One tile of rows; VEC elements per access.  Dim 0 has stride 1 in A and B
// whenever VEC > 1 (checked by the planner).
template <typename E, int MODE, bool UPD, typename OffT, int VEC>
__device__ __forceinline__ void rows_body(const HpttProblem &P, const HpttTile &T,
                                          const E *__restrict__ A, E *__restrict__ B,
                                          const Op<E, MODE, UPD> &op,
                                          const RowThread<OffT> &s, const TileOrigin &o,
                                          const OffT *tInY, const OffT *tOutY,
                                          const int *tCy) {
  if (!s.active) return;
  constexpr int kJMax = hptt_jmax_rows(sizeof(E) * VEC);
  const int64_t col = static_cast<int64_t>(s.e) * VEC;
  const bool col_ok = o.interior || col < o.remX;
  const E *src = A + o.bA + col * P.sA[0];
  E *dst = B + o.bB + col * P.sB[0];
  Vec<E, VEC> av[kJMax];
  Vec<E, VEC> bv[kJMax];
#pragma unroll
  for (int j = 0; j < kJMax; ++j) {
    const int y = s.y0 + j * T.R1;
    if (j < T.J1 && y < T.TY && col_ok && (o.interior || tCy[y] < o.remY)) {
      av[j] = ld_vec<E, VEC>(src + tInY[y]);
      if (UPD) bv[j] = ld_vec_rw<E, VEC>(dst + tOutY[y]);
    }
  }
#pragma unroll
  for (int j = 0; j < kJMax; ++j) {
    const int y = s.y0 + j * T.R1;
    if (j < T.J1 && y < T.TY && col_ok && (o.interior || tCy[y] < o.remY)) {
      Vec<E, VEC> r;
#pragma unroll
      for (int k = 0; k < VEC; ++k) r.v[k] = op(av[j].v[k], UPD ? bv[j].v[k] : av[j].v[k]);
      st_vec<E, VEC>(dst + tOutY[y], r, !UPD);
    }
  }
}

__host__ __device__ inline int align16(int x) { return (x + 15) & ~15; }

}  // namespace dev
}  // namespace hptt_b200
