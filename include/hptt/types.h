// Public types of the hptt C++ interface (B200 build).
//
// Same names and meanings as the reference's inc/hptt/types.h:14-54, so code
// written against the reference compiles unchanged: index aliases, the two
// complex element types (C99 _Complex, layout-compatible with float2 /
// double2 on the device) and DeducedFloatType, the scalar type of alpha and
// beta (the element's real type: complex elements take REAL scalars, applied
// to both components).
#pragma once
#ifndef HPTT_TYPES_H_
#define HPTT_TYPES_H_

#include <cstdint>

namespace hptt {

using TensorIdx = uint64_t;
using TensorInt = int32_t;
using TensorUInt = uint32_t;

using FloatComplex = float _Complex;
using DoubleComplex = double _Complex;

template <typename FloatType>
struct FloatTypeDeducer;
template <>
struct FloatTypeDeducer<float> {
  using type = float;
};
template <>
struct FloatTypeDeducer<double> {
  using type = double;
};
template <>
struct FloatTypeDeducer<FloatComplex> {
  using type = float;
};
template <>
struct FloatTypeDeducer<DoubleComplex> {
  using type = double;
};

template <typename FloatType>
using DeducedFloatType = typename FloatTypeDeducer<FloatType>::type;

}  // namespace hptt

#endif  // HPTT_TYPES_H_
