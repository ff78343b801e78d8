// Harness that drives the reference's OWN CPU transpose plan, compiled from
// the reference sources by oracle/Makefile into oracle/_ref/libhptt_ref.so.
// TEST INFRASTRUCTURE ONLY: used to pin the oracle restatement and as the
// timed CPU baseline.  The product never links it.
//
// The reference's CMake code generator is not run.  In its place this file
// builds the plan the same way the generated plan package does
// (cmake/pylib/gen_util/hptt_trans_gen.py:174-201): input/output
// TensorWrapper with out_size[i] = in_size[perm[i]], ParamTrans with
// UPDATE = |beta| >= 1e-16 (inc/hptt/impl/hptt_trans_impl.h:75-78), PlanTrans
// with heuristic budget 5040 and tuning budget 64 when tuning_timeout != 0
// (inc/hptt/impl/hptt_trans_impl.h:90-102), then CGraphTrans::exec.
// Outer sizes are not exposed: the reference drops in_outer_size
// (hptt_trans_gen.py:189), so only dense tensors are driven here.
//
// hptt_ref_naive runs the reference's naive OpenMP transpose RefTrans
// (test/inc/hptt/test_util.tcc:143-185), which is what the reference's own
// benchmark compares against and what is timed on shapes where the plan is
// known to be incorrect.
#include <hptt/types.h>
#include <hptt/tensor.h>
#include <hptt/param/parameter_trans.h>
#include <hptt/plan/plan_trans.h>
#include <hptt/cgraph/cgraph_trans.h>
#include <hptt/test_util.h>

#include <omp.h>

#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <memory>
#include <vector>

namespace {

using hptt::TensorIdx;
using hptt::TensorUInt;

template <typename T, TensorUInt ORDER, bool UPDATE>
struct RefRunner {
  using Param = hptt::ParamTrans<hptt::TensorWrapper<T, ORDER>, UPDATE>;
  using Graph = hptt::CGraphTrans<Param>;

  static int run(const T *in, T *out, const uint32_t *in_size,
                 const uint32_t *perm, hptt::DeducedFloatType<T> alpha,
                 hptt::DeducedFloatType<T> beta, uint32_t threads,
                 double tuning_timeout, int repeat, double *best_s) {
    std::vector<TensorIdx> in_vec(in_size, in_size + ORDER), out_vec(ORDER);
    std::array<TensorUInt, ORDER> perm_arr;
    for (TensorUInt k = 0; k < ORDER; ++k) {
      out_vec[k] = in_vec[perm[k]];
      perm_arr[k] = perm[k];
    }
    hptt::TensorSize<ORDER> in_sz(in_vec), out_sz(out_vec);
    const hptt::TensorWrapper<T, ORDER> in_t(in_sz, in_sz, in);
    hptt::TensorWrapper<T, ORDER> out_t(out_sz, out_sz, out);
    const int tune = tuning_timeout == 0.0 ? 0 : 64;
    hptt::PlanTrans<Param> plan(
        std::make_shared<Param>(in_t, out_t, perm_arr, alpha, beta), threads,
        tune, tune, 5040, 5040, tuning_timeout * 1000.0);
    std::unique_ptr<Graph> graph(plan.get_graph());
    double best = 1e300;
    for (int r = 0; r < (repeat < 1 ? 1 : repeat); ++r) {
      auto t0 = std::chrono::steady_clock::now();
      graph->exec();
      auto t1 = std::chrono::steady_clock::now();
      double s = std::chrono::duration<double>(t1 - t0).count();
      if (s < best) best = s;
    }
    if (best_s) *best_s = best;
    return 0;
  }
};

template <typename T, TensorUInt ORDER>
int run_order(const void *in, void *out, const uint32_t *in_size,
              const uint32_t *perm, double alpha, double beta,
              uint32_t threads, double timeout, int repeat, double *best) {
  using D = hptt::DeducedFloatType<T>;
  const D a = static_cast<D>(alpha), b = static_cast<D>(beta);
  if (std::fabs(b) >= 1e-16)
    return RefRunner<T, ORDER, true>::run(
        static_cast<const T *>(in), static_cast<T *>(out), in_size, perm, a,
        b, threads, timeout, repeat, best);
  return RefRunner<T, ORDER, false>::run(
      static_cast<const T *>(in), static_cast<T *>(out), in_size, perm, a, b,
      threads, timeout, repeat, best);
}

template <typename T>
int run_type(int rank, const void *in, void *out, const uint32_t *in_size,
             const uint32_t *perm, double alpha, double beta, uint32_t threads,
             double timeout, int repeat, double *best) {
  switch (rank) {
    case 2: return run_order<T, 2>(in, out, in_size, perm, alpha, beta, threads, timeout, repeat, best);
    case 3: return run_order<T, 3>(in, out, in_size, perm, alpha, beta, threads, timeout, repeat, best);
    case 4: return run_order<T, 4>(in, out, in_size, perm, alpha, beta, threads, timeout, repeat, best);
    case 5: return run_order<T, 5>(in, out, in_size, perm, alpha, beta, threads, timeout, repeat, best);
    case 6: return run_order<T, 6>(in, out, in_size, perm, alpha, beta, threads, timeout, repeat, best);
    default: return -1;
  }
}

template <typename T>
int naive_type(int rank, const void *in, void *out, const uint32_t *in_size,
               const uint32_t *perm, double alpha, double beta, int repeat,
               double *best_s) {
  using D = hptt::DeducedFloatType<T>;
  std::vector<TensorIdx> size(in_size, in_size + rank);
  std::vector<TensorUInt> p(perm, perm + rank);
  hptt::RefTrans<T> ref;
  double best = 1e300;
  for (int r = 0; r < (repeat < 1 ? 1 : repeat); ++r) {
    auto t0 = std::chrono::steady_clock::now();
    ref(static_cast<const T *>(in), static_cast<T *>(out), size, p,
        static_cast<D>(alpha), static_cast<D>(beta));
    auto t1 = std::chrono::steady_clock::now();
    double s = std::chrono::duration<double>(t1 - t0).count();
    if (s < best) best = s;
  }
  if (best_s) *best_s = best;
  return 0;
}

}  // namespace

extern "C" {

// dtype: 0 f32, 1 f64, 2 c64, 3 c128.  Dense tensors, real scalars.
// Runs create-plan + exec `repeat` times (exec only is timed); returns 0 on
// success.  `best_seconds` receives the fastest exec.
int hptt_ref_plan_exec(int dtype, int rank, const uint32_t *in_size,
                       const uint32_t *perm, double alpha, double beta,
                       const void *in, void *out, uint32_t threads,
                       double tuning_timeout, int repeat,
                       double *best_seconds) {
  switch (dtype) {
    case 0: return run_type<float>(rank, in, out, in_size, perm, alpha, beta, threads, tuning_timeout, repeat, best_seconds);
    case 1: return run_type<double>(rank, in, out, in_size, perm, alpha, beta, threads, tuning_timeout, repeat, best_seconds);
    case 2: return run_type<hptt::FloatComplex>(rank, in, out, in_size, perm, alpha, beta, threads, tuning_timeout, repeat, best_seconds);
    case 3: return run_type<hptt::DoubleComplex>(rank, in, out, in_size, perm, alpha, beta, threads, tuning_timeout, repeat, best_seconds);
    default: return -1;
  }
}

// The reference's naive OpenMP transpose (always reads B).
int hptt_ref_naive_exec(int dtype, int rank, const uint32_t *in_size,
                        const uint32_t *perm, double alpha, double beta,
                        const void *in, void *out, uint32_t threads,
                        int repeat, double *best_seconds) {
  if (threads > 0) omp_set_num_threads(static_cast<int>(threads));
  switch (dtype) {
    case 0: return naive_type<float>(rank, in, out, in_size, perm, alpha, beta, repeat, best_seconds);
    case 1: return naive_type<double>(rank, in, out, in_size, perm, alpha, beta, repeat, best_seconds);
    case 2: return naive_type<hptt::FloatComplex>(rank, in, out, in_size, perm, alpha, beta, repeat, best_seconds);
    case 3: return naive_type<hptt::DoubleComplex>(rank, in, out, in_size, perm, alpha, beta, repeat, best_seconds);
    default: return -1;
  }
}

int hptt_ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
