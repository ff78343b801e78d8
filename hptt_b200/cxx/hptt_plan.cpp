// C++14 host side of the hptt interface (include/hptt/hptt.h) over the C ABI
// of libhptt_cuda.so.  Built as libhptt.so; links libhptt_cuda.so.
//
// create_plan keeps the reference's contract (src/hptt.cc:16-93): the same
// argument guard with nullptr on failure, a shared_ptr the caller owns, and a
// plan that never owns or frees the data.  Where the reference dlopens an
// architecture library and resolves create_trans_plan_impl_{s,d,c,z}, this
// library defines those factories itself and they call the GPU engine.
#include <hptt/hptt.h>

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "hptt_cuda.h"

namespace hptt {
namespace {

template <typename T> struct DtypeOf;
template <> struct DtypeOf<float> { static constexpr int value = HPTT_CUDA_F32; };
template <> struct DtypeOf<double> { static constexpr int value = HPTT_CUDA_F64; };
template <> struct DtypeOf<FloatComplex> { static constexpr int value = HPTT_CUDA_C64; };
template <> struct DtypeOf<DoubleComplex> { static constexpr int value = HPTT_CUDA_C128; };

// One plan: owns the C ABI handle, never the data.
template <typename T>
class GpuTransPlan final : public CudaTransPlan<T> {
 public:
  explicit GpuTransPlan(hptt_cuda_plan_t h) : h_(h) {}
  ~GpuTransPlan() override { hptt_cuda_plan_destroy(h_); }

  void exec() override { status_ = hptt_cuda_plan_exec(h_); }
  void operator()() override { exec(); }
  void print_plan() override {
    const std::string s = describe();
    std::fwrite(s.data(), 1, s.size(), stdout);
    std::fflush(stdout);
  }
  void reset_data(const T *in_data, T *out_data) override {
    hptt_cuda_plan_reset_data(h_, in_data, out_data);
  }
  void set_thread_ids(const std::vector<int32_t> &ids) override {
    hptt_cuda_plan_set_thread_ids(h_, ids.data(), static_cast<uint32_t>(ids.size()));
  }
  void unset_thread_ids() override { hptt_cuda_plan_unset_thread_ids(h_); }

  int sync() override { return hptt_cuda_plan_sync(h_); }
  int set_stream(void *stream) override { return hptt_cuda_plan_set_stream(h_, stream); }
  int exec_on(void *stream) override { return status_ = hptt_cuda_plan_exec_on(h_, stream); }
  int status() const override { return status_; }
  int set_coef(DeducedFloatType<T> alpha, DeducedFloatType<T> beta) override {
    const double a[2] = {static_cast<double>(alpha), 0.0};
    const double b[2] = {static_cast<double>(beta), 0.0};
    return hptt_cuda_plan_set_coef(h_, a, b, 0);
  }
  std::string describe() const override {
    std::vector<char> buf(8192, '\0');
    if (hptt_cuda_plan_describe(h_, buf.data(), buf.size()) != HPTT_OK) return std::string();
    return std::string(buf.data());
  }
  uint64_t bytes() const override {
    uint64_t b = 0;
    hptt_cuda_plan_bytes(h_, &b);
    return b;
  }

 private:
  hptt_cuda_plan_t h_;
  int status_ = HPTT_OK;
};

// The reference's guard on the vector arguments (src/hptt.cc:25-56) that the
// C ABI cannot see (it takes raw arrays of length `order`); the value checks
// (zero extents, outer sizes, the permutation) are the C ABI's.
bool vectors_ok(uint32_t order, const std::vector<uint32_t> &in_size,
                const std::vector<uint32_t> &perm, const std::vector<uint32_t> &in_outer,
                const std::vector<uint32_t> &out_outer) {
  if (order <= 1) return false;
  if (in_size.size() != order || perm.size() != order) return false;
  if (!in_outer.empty() && in_outer.size() != order) return false;
  if (!out_outer.empty() && out_outer.size() != order) return false;
  return true;
}

template <typename T>
GpuTransPlan<T> *make_plan(const T *in_data, T *out_data, uint32_t order,
                           const std::vector<uint32_t> &in_size,
                           const std::vector<uint32_t> &perm, const double alpha[2],
                           const double beta[2], int complex_scalars, uint32_t num_threads,
                           double tuning_timeout, const std::vector<uint32_t> &in_outer,
                           const std::vector<uint32_t> &out_outer) {
  if (in_data == nullptr || out_data == nullptr) return nullptr;
  if (!vectors_ok(order, in_size, perm, in_outer, out_outer)) return nullptr;
  hptt_cuda_plan_t h = nullptr;
  const int st = hptt_cuda_plan_create(
      DtypeOf<T>::value, order, in_size.data(), perm.data(),
      in_outer.empty() ? nullptr : in_outer.data(),
      out_outer.empty() ? nullptr : out_outer.data(), alpha, beta, complex_scalars, in_data,
      out_data, num_threads, tuning_timeout, &h);
  if (st != HPTT_OK || h == nullptr) return nullptr;
  GpuTransPlan<T> *p = new (std::nothrow) GpuTransPlan<T>(h);
  if (p == nullptr) hptt_cuda_plan_destroy(h);
  return p;
}

template <typename T>
CGraphTransPackBase<T> *factory(const T *in_data, T *out_data, uint32_t order,
                                const std::vector<uint32_t> &in_size,
                                const std::vector<uint32_t> &perm, DeducedFloatType<T> alpha,
                                DeducedFloatType<T> beta, uint32_t num_threads,
                                double tuning_timeout, const std::vector<uint32_t> &in_outer,
                                const std::vector<uint32_t> &out_outer) {
  const double a[2] = {static_cast<double>(alpha), 0.0};
  const double b[2] = {static_cast<double>(beta), 0.0};
  return make_plan<T>(in_data, out_data, order, in_size, perm, a, b, 0, num_threads,
                      tuning_timeout, in_outer, out_outer);
}

}  // namespace

template <typename FloatType>
std::shared_ptr<trans_plan<FloatType>> create_plan(
    const FloatType *in_data, FloatType *out_data, const std::vector<uint32_t> &in_size,
    const std::vector<uint32_t> &perm, const DeducedFloatType<FloatType> alpha,
    const DeducedFloatType<FloatType> beta, const uint32_t num_threads,
    const double tuning_timeout, const std::vector<uint32_t> &in_outer_size,
    const std::vector<uint32_t> &out_outer_size) {
  return std::shared_ptr<trans_plan<FloatType>>(
      factory<FloatType>(in_data, out_data, static_cast<uint32_t>(perm.size()), in_size,
                         perm, alpha, beta, num_threads, tuning_timeout, in_outer_size,
                         out_outer_size));
}

template std::shared_ptr<trans_plan<float>> create_plan<float>(
    const float *, float *, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &,
    const float, const float, const TensorUInt, const double,
    const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);
template std::shared_ptr<trans_plan<double>> create_plan<double>(
    const double *, double *, const std::vector<TensorUInt> &,
    const std::vector<TensorUInt> &, const double, const double, const TensorUInt,
    const double, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);
template std::shared_ptr<trans_plan<FloatComplex>> create_plan<FloatComplex>(
    const FloatComplex *, FloatComplex *, const std::vector<TensorUInt> &,
    const std::vector<TensorUInt> &, const float, const float, const TensorUInt,
    const double, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);
template std::shared_ptr<trans_plan<DoubleComplex>> create_plan<DoubleComplex>(
    const DoubleComplex *, DoubleComplex *, const std::vector<TensorUInt> &,
    const std::vector<TensorUInt> &, const double, const double, const TensorUInt,
    const double, const std::vector<TensorUInt> &, const std::vector<TensorUInt> &);

std::shared_ptr<trans_plan<FloatComplex>> create_plan(
    const FloatComplex *in_data, FloatComplex *out_data, const std::vector<uint32_t> &in_size,
    const std::vector<uint32_t> &perm, std::complex<float> alpha, std::complex<float> beta,
    const uint32_t num_threads, const double tuning_timeout,
    const std::vector<uint32_t> &in_outer_size, const std::vector<uint32_t> &out_outer_size) {
  const double a[2] = {alpha.real(), alpha.imag()};
  const double b[2] = {beta.real(), beta.imag()};
  return std::shared_ptr<trans_plan<FloatComplex>>(make_plan<FloatComplex>(
      in_data, out_data, static_cast<uint32_t>(perm.size()), in_size, perm, a, b, 1,
      num_threads, tuning_timeout, in_outer_size, out_outer_size));
}

std::shared_ptr<trans_plan<DoubleComplex>> create_plan(
    const DoubleComplex *in_data, DoubleComplex *out_data,
    const std::vector<uint32_t> &in_size, const std::vector<uint32_t> &perm,
    std::complex<double> alpha, std::complex<double> beta, const uint32_t num_threads,
    const double tuning_timeout, const std::vector<uint32_t> &in_outer_size,
    const std::vector<uint32_t> &out_outer_size) {
  const double a[2] = {alpha.real(), alpha.imag()};
  const double b[2] = {beta.real(), beta.imag()};
  return std::shared_ptr<trans_plan<DoubleComplex>>(make_plan<DoubleComplex>(
      in_data, out_data, static_cast<uint32_t>(perm.size()), in_size, perm, a, b, 1,
      num_threads, tuning_timeout, in_outer_size, out_outer_size));
}

}  // namespace hptt

hptt::CGraphTransPackBase<float> *create_trans_plan_impl_s(
    const float *in_data, float *out_data, const hptt::TensorUInt order,
    const std::vector<hptt::TensorUInt> &in_size, const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<float> alpha, const hptt::DeducedFloatType<float> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size) {
  return hptt::factory<float>(in_data, out_data, order, in_size, perm, alpha, beta,
                              num_threads, tuning_timeout, in_outer_size, out_outer_size);
}

hptt::CGraphTransPackBase<double> *create_trans_plan_impl_d(
    const double *in_data, double *out_data, const hptt::TensorUInt order,
    const std::vector<hptt::TensorUInt> &in_size, const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<double> alpha, const hptt::DeducedFloatType<double> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size) {
  return hptt::factory<double>(in_data, out_data, order, in_size, perm, alpha, beta,
                               num_threads, tuning_timeout, in_outer_size, out_outer_size);
}

hptt::CGraphTransPackBase<hptt::FloatComplex> *create_trans_plan_impl_c(
    const hptt::FloatComplex *in_data, hptt::FloatComplex *out_data,
    const hptt::TensorUInt order, const std::vector<hptt::TensorUInt> &in_size,
    const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<hptt::FloatComplex> alpha,
    const hptt::DeducedFloatType<hptt::FloatComplex> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size) {
  return hptt::factory<hptt::FloatComplex>(in_data, out_data, order, in_size, perm, alpha,
                                           beta, num_threads, tuning_timeout, in_outer_size,
                                           out_outer_size);
}

hptt::CGraphTransPackBase<hptt::DoubleComplex> *create_trans_plan_impl_z(
    const hptt::DoubleComplex *in_data, hptt::DoubleComplex *out_data,
    const hptt::TensorUInt order, const std::vector<hptt::TensorUInt> &in_size,
    const std::vector<hptt::TensorUInt> &perm,
    const hptt::DeducedFloatType<hptt::DoubleComplex> alpha,
    const hptt::DeducedFloatType<hptt::DoubleComplex> beta,
    const hptt::TensorUInt num_threads, const double tuning_timeout,
    const std::vector<hptt::TensorUInt> &in_outer_size,
    const std::vector<hptt::TensorUInt> &out_outer_size) {
  return hptt::factory<hptt::DoubleComplex>(in_data, out_data, order, in_size, perm, alpha,
                                            beta, num_threads, tuning_timeout,
                                            in_outer_size, out_outer_size);
}
