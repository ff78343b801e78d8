// Tensor contraction through hptt transposes (C++ interface, header-only over
// the C ABI of libhptt_cuda.so; link with -lhptt_cuda).
//
//   C[labels_c] = alpha * sum_K A[labels_a] * B[labels_b] + beta * C[labels_c]
//
// No counterpart in the reference, which only transposes: this is the
// transpose - GEMM - transpose sequence contraction code builds from
// create_plan/exec/reset_data (reference README.md:48-72), as one plan.
// Tensors are dense, column-major (first extent has stride 1) DEVICE
// buffers; a label (any int32) appears at most once per tensor; C's extents
// come from A and B.  create_contraction returns nullptr where the C ABI
// reports an error (invalid labels, sizes, no device, allocation), in the
// style of hptt::create_plan.  exec() is asynchronous on the plan's stream.
#pragma once
#ifndef HPTT_CONTRACTION_H_
#define HPTT_CONTRACTION_H_

#include <complex>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include <hptt/types.h>
#include <hptt_cuda.h>

namespace hptt {

template <typename T>
struct ContractDtype;
template <>
struct ContractDtype<float> {
  static constexpr int value = HPTT_CUDA_F32;
};
template <>
struct ContractDtype<double> {
  static constexpr int value = HPTT_CUDA_F64;
};
template <>
struct ContractDtype<FloatComplex> {
  static constexpr int value = HPTT_CUDA_C64;
};
template <>
struct ContractDtype<DoubleComplex> {
  static constexpr int value = HPTT_CUDA_C128;
};

template <typename T>
class contraction_plan {
 public:
  explicit contraction_plan(hptt_cuda_contract_t h) : h_(h) {}
  ~contraction_plan() { hptt_cuda_contract_destroy(h_); }
  contraction_plan(const contraction_plan &) = delete;
  contraction_plan &operator=(const contraction_plan &) = delete;

  // Enqueue on the plan's stream (legacy default stream unless set_stream).
  int exec() { return hptt_cuda_contract_exec(h_); }
  int operator()() { return exec(); }
  // Enqueue on a cudaStream_t passed as void*.
  int exec_on(void *stream) { return hptt_cuda_contract_exec_on(h_, stream); }
  int reset_data(const T *A, const T *B, T *C) {
    return hptt_cuda_contract_reset_data(h_, A, B, C);
  }
  int set_stream(void *stream) { return hptt_cuda_contract_set_stream(h_, stream); }
  int set_graph(bool on) { return hptt_cuda_contract_set_graph(h_, on ? 1 : 0); }
  int sync() { return hptt_cuda_contract_sync(h_); }
  hptt_cuda_contract_stats info() const {
    hptt_cuda_contract_stats s{};
    hptt_cuda_contract_info(h_, &s);
    return s;
  }
  std::string describe() const {
    char buf[4096];
    if (hptt_cuda_contract_describe(h_, buf, sizeof(buf)) != HPTT_OK) return std::string();
    return std::string(buf);
  }
  void print_plan() const { std::fputs(describe().c_str(), stdout); }

 private:
  hptt_cuda_contract_t h_;
};

namespace detail {
template <typename T>
std::shared_ptr<contraction_plan<T>> create_contraction_(
    const T *A, const std::vector<uint32_t> &size_a, const std::vector<int32_t> &labels_a,
    const T *B, const std::vector<uint32_t> &size_b, const std::vector<int32_t> &labels_b,
    T *C, const std::vector<int32_t> &labels_c, const double *alpha, const double *beta,
    int complex_scalars, void *workspace, uint64_t workspace_bytes) {
  if (size_a.size() != labels_a.size() || size_b.size() != labels_b.size()) return nullptr;
  hptt_cuda_contract_t h = nullptr;
  const int st = hptt_cuda_contract_create(
      ContractDtype<T>::value, static_cast<uint32_t>(size_a.size()), size_a.data(),
      labels_a.data(), static_cast<uint32_t>(size_b.size()), size_b.data(), labels_b.data(),
      static_cast<uint32_t>(labels_c.size()), labels_c.empty() ? nullptr : labels_c.data(),
      alpha, beta, complex_scalars, A, B, C, workspace, workspace_bytes, &h);
  if (st != HPTT_OK || !h) return nullptr;
  return std::make_shared<contraction_plan<T>>(h);
}
}  // namespace detail

// Real scalars (complex element types scale both components, as the
// transposes do).
template <typename T>
std::shared_ptr<contraction_plan<T>> create_contraction(
    const T *A, const std::vector<uint32_t> &size_a, const std::vector<int32_t> &labels_a,
    const T *B, const std::vector<uint32_t> &size_b, const std::vector<int32_t> &labels_b,
    T *C, const std::vector<int32_t> &labels_c, const DeducedFloatType<T> alpha,
    const DeducedFloatType<T> beta, void *workspace = nullptr, uint64_t workspace_bytes = 0) {
  const double al[2] = {static_cast<double>(alpha), 0.0};
  const double be[2] = {static_cast<double>(beta), 0.0};
  return detail::create_contraction_<T>(A, size_a, labels_a, B, size_b, labels_b, C, labels_c,
                                        al, be, 0, workspace, workspace_bytes);
}

// Complex scalars for complex element types.
template <typename T>
std::shared_ptr<contraction_plan<T>> create_contraction(
    const T *A, const std::vector<uint32_t> &size_a, const std::vector<int32_t> &labels_a,
    const T *B, const std::vector<uint32_t> &size_b, const std::vector<int32_t> &labels_b,
    T *C, const std::vector<int32_t> &labels_c, std::complex<DeducedFloatType<T>> alpha,
    std::complex<DeducedFloatType<T>> beta, void *workspace = nullptr,
    uint64_t workspace_bytes = 0) {
  const double al[2] = {static_cast<double>(alpha.real()), static_cast<double>(alpha.imag())};
  const double be[2] = {static_cast<double>(beta.real()), static_cast<double>(beta.imag())};
  return detail::create_contraction_<T>(A, size_a, labels_a, B, size_b, labels_b, C, labels_c,
                                        al, be, 1, workspace, workspace_bytes);
}

}  // namespace hptt

#endif  // HPTT_CONTRACTION_H_
