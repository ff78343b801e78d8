// Element arithmetic of B = alpha * A(perm) + beta * B, bit-compatible with
// the reference's CPU kernels.
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

}  // namespace dev
}  // namespace hptt_b200
