// hptt C++ interface, B200 build (libhptt.so over libhptt_cuda.so).
//
//   B[perm(i)] = alpha * A[i] + beta * B[perm(i)]
//
// A drop-in for the reference's public header (inc/hptt/hptt.h:85-123): the
// same create_plan template, signature, defaults and nullptr-on-error rule,
// explicitly instantiated for float, double, FloatComplex and DoubleComplex.
// Differences, all on the device side:
//   * in_data / out_data are DEVICE pointers (cudaMalloc'd or managed);
//   * exec() is asynchronous on the plan's CUDA stream (see
//     impl/hptt_trans.h for sync() and the other extensions);
//   * num_threads is accepted and ignored; tuning_timeout != 0 times
//     candidate tile shapes on the GPU (< 0: all, > 0: at most that many
//     seconds) and caches the winner per (dtype, rank, perm, size class).
// create_plan returns nullptr when the reference does (src/hptt.cc:25-56):
// a null data pointer, rank < 2, size vectors of the wrong length, a zero
// extent or an outer size below the extent, an invalid permutation -- and
// also when no CUDA device is usable or the plan cannot be built.
#pragma once
#ifndef HPTT_HPTT_H_
#define HPTT_HPTT_H_

#include <complex>
#include <cstdint>
#include <memory>
#include <vector>

#include <hptt/impl/hptt_trans.h>
#include <hptt/types.h>

namespace hptt {

template <typename FloatType>
std::shared_ptr<trans_plan<FloatType>> create_plan(
    const FloatType *in_data, FloatType *out_data, const std::vector<uint32_t> &in_size,
    const std::vector<uint32_t> &perm, const DeducedFloatType<FloatType> alpha,
    const DeducedFloatType<FloatType> beta, const uint32_t num_threads,
    const double tuning_timeout = 0.0, const std::vector<uint32_t> &in_outer_size = {},
    const std::vector<uint32_t> &out_outer_size = {});

extern template std::shared_ptr<trans_plan<float>> create_plan<float>(
    const float *, float *, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &,
    const float, const float, const TensorUInt, const double,
    const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);
extern template std::shared_ptr<trans_plan<double>> create_plan<double>(
    const double *, double *, const std::vector<TensorUInt> &,
    const std::vector<TensorUInt> &, const double, const double, const TensorUInt,
    const double, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);
extern template std::shared_ptr<trans_plan<FloatComplex>> create_plan<FloatComplex>(
    const FloatComplex *, FloatComplex *, const std::vector<TensorUInt> &,
    const std::vector<TensorUInt> &, const float, const float, const TensorUInt,
    const double, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);
extern template std::shared_ptr<trans_plan<DoubleComplex>> create_plan<DoubleComplex>(
    const DoubleComplex *, DoubleComplex *, const std::vector<TensorUInt> &,
    const std::vector<TensorUInt> &, const double, const double, const TensorUInt,
    const double, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);

// Extension: complex alpha and beta for complex elements (the reference
// takes real scalars only).  Products are rounded as
//   re = fl(fl(sr*xr) - fl(si*xi)),  im = fl(fl(sr*xi) + fl(si*xr))
// without FMA, then out = fl(alpha*a + beta*b) componentwise.
std::shared_ptr<trans_plan<FloatComplex>> create_plan(
    const FloatComplex *in_data, FloatComplex *out_data, const std::vector<uint32_t> &in_size,
    const std::vector<uint32_t> &perm, std::complex<float> alpha, std::complex<float> beta,
    const uint32_t num_threads, const double tuning_timeout = 0.0,
    const std::vector<uint32_t> &in_outer_size = {},
    const std::vector<uint32_t> &out_outer_size = {});
std::shared_ptr<trans_plan<DoubleComplex>> create_plan(
    const DoubleComplex *in_data, DoubleComplex *out_data,
    const std::vector<uint32_t> &in_size, const std::vector<uint32_t> &perm,
    std::complex<double> alpha, std::complex<double> beta, const uint32_t num_threads,
    const double tuning_timeout = 0.0, const std::vector<uint32_t> &in_outer_size = {},
    const std::vector<uint32_t> &out_outer_size = {});

}  // namespace hptt

// The per-type factories the reference's loader resolves by their mangled
// names (src/hptt.cc:58-92, src/impl/hptt_trans_impl_s.cc:8-20).  They take
// the rank as `order` and return a plan the caller owns (nullptr on error).
hptt::CGraphTransPackBase<float> *create_trans_plan_impl_s(
    const float *in_data, float *out_data, const hptt::TensorUInt order,
    const std::vector<hptt::TensorUInt> &in_size, const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<float> alpha, const hptt::DeducedFloatType<float> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size);
hptt::CGraphTransPackBase<double> *create_trans_plan_impl_d(
    const double *in_data, double *out_data, const hptt::TensorUInt order,
    const std::vector<hptt::TensorUInt> &in_size, const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<double> alpha, const hptt::DeducedFloatType<double> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size);
hptt::CGraphTransPackBase<hptt::FloatComplex> *create_trans_plan_impl_c(
    const hptt::FloatComplex *in_data, hptt::FloatComplex *out_data,
    const hptt::TensorUInt order, const std::vector<hptt::TensorUInt> &in_size,
    const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<hptt::FloatComplex> alpha,
    const hptt::DeducedFloatType<hptt::FloatComplex> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size);
hptt::CGraphTransPackBase<hptt::DoubleComplex> *create_trans_plan_impl_z(
    const hptt::DoubleComplex *in_data, hptt::DoubleComplex *out_data,
    const hptt::TensorUInt order, const std::vector<hptt::TensorUInt> &in_size,
    const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<hptt::DoubleComplex> alpha,
    const hptt::DeducedFloatType<hptt::DoubleComplex> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size);

#endif  // HPTT_HPTT_H_
