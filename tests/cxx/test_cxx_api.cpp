// Test program for the C++ interface (include/hptt/hptt.h, libhptt.so),
// written the way a user of the reference API writes it.  Run by
// tests/test_cxx_api.py.
//
//   test_cxx_api guard   no device needed: the argument guard returns
//                        nullptr exactly where the reference's does
//                        (src/hptt.cc:25-56)
//   test_cxx_api gpu     every element type through create_plan / exec /
//                        reset_data / the complex-scalar overload and the
//                        create_trans_plan_impl_* factories (resolved by
//                        their mangled names with dlsym, as the reference's
//                        loader does), each result compared bit for bit with
//                        the oracle (the CPU restatement in oracle/).
// Exit status 0 when every check passes.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <hptt/contraction.h>
#include <hptt/hptt.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "oracle.h"

namespace {

int g_fail = 0;

void check(bool ok, const std::string &what) {
  if (!ok) {
    std::printf("FAIL %s\n", what.c_str());
    ++g_fail;
  }
}

template <typename T> struct Code;
template <> struct Code<float> { static constexpr int v = 0; };
template <> struct Code<double> { static constexpr int v = 1; };
template <> struct Code<hptt::FloatComplex> { static constexpr int v = 2; };
template <> struct Code<hptt::DoubleComplex> { static constexpr int v = 3; };

template <typename T>
std::vector<T> random_tensor(size_t n, std::mt19937_64 &rng) {
  using R = hptt::DeducedFloatType<T>;
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  const size_t comps = sizeof(T) / sizeof(R);
  std::vector<T> v(n);
  R *p = reinterpret_cast<R *>(v.data());
  for (size_t i = 0; i < n * comps; ++i) p[i] = static_cast<R>(u(rng));
  return v;
}

size_t prod(const std::vector<uint32_t> &v) {
  size_t n = 1;
  for (uint32_t x : v) n *= x;
  return n;
}

// ---------------------------------------------------------------------------
int run_guard() {
  // Non-null stand-ins: every call below fails its guard before any data
  // pointer is used.
  float dummy_in[1] = {0.0f}, dummy_out[1] = {0.0f};
  const float *in = dummy_in;
  float *out = dummy_out;
  const std::vector<uint32_t> size{4, 5, 6}, perm{2, 0, 1};
  check(hptt::create_plan<float>(nullptr, out, size, perm, 1.0f, 0.0f, 1) == nullptr,
        "null input");
  check(hptt::create_plan<float>(in, nullptr, size, perm, 1.0f, 0.0f, 1) == nullptr,
        "null output");
  check(hptt::create_plan<float>(in, out, {4}, {0}, 1.0f, 0.0f, 1) == nullptr, "rank 1");
  check(hptt::create_plan<float>(in, out, {4, 5}, perm, 1.0f, 0.0f, 1) == nullptr,
        "in_size length");
  check(hptt::create_plan<float>(in, out, {4, 0, 6}, perm, 1.0f, 0.0f, 1) == nullptr,
        "zero extent");
  check(hptt::create_plan<float>(in, out, size, {2, 2, 1}, 1.0f, 0.0f, 1) == nullptr,
        "repeated perm index");
  check(hptt::create_plan<float>(in, out, size, {3, 0, 1}, 1.0f, 0.0f, 1) == nullptr,
        "perm index out of range");
  check(hptt::create_plan<float>(in, out, size, perm, 1.0f, 0.0f, 1, 0.0, {4, 5}) == nullptr,
        "in_outer length");
  check(hptt::create_plan<float>(in, out, size, perm, 1.0f, 0.0f, 1, 0.0, {4, 4, 6}) ==
            nullptr,
        "in_outer below extent");
  check(hptt::create_plan<float>(in, out, size, perm, 1.0f, 0.0f, 1, 0.0, {}, {6, 4}) ==
            nullptr,
        "out_outer length");
  // contraction (include/hptt/contraction.h): invalid labels fail before any
  // device work
  float dummy_c[1] = {0.0f};
  check(hptt::create_contraction<float>(in, {3, 4}, {'i', 'k'}, in, {5, 2}, {'k', 'j'}, dummy_c,
                                        {'i', 'j'}, 1.0f, 0.0f) == nullptr,
        "contraction: K extents differ");
  check(hptt::create_contraction<float>(in, {3, 4}, {'i', 'k'}, in, {4, 2}, {'k', 'j'}, dummy_c,
                                        {'i'}, 1.0f, 0.0f) == nullptr,
        "contraction: j summed over B alone");
  check(hptt::create_contraction<float>(in, {3, 3}, {'i', 'i'}, in, {3}, {'i'}, dummy_c, {'i'},
                                        1.0f, 0.0f) == nullptr,
        "contraction: repeated label");
  // factories: same guard, raw pointer result
  check(create_trans_plan_impl_s(in, out, 1, {4}, {0}, 1.0f, 0.0f, 1, 0.0, {}, {}) == nullptr,
        "factory rank 1");
  check(create_trans_plan_impl_d(nullptr, nullptr, 2, {4, 5}, {1, 0}, 1.0, 0.0, 1, 0.0, {},
                                 {}) == nullptr,
        "factory null data");
  std::printf("guard checks done, %d failure(s)\n", g_fail);
  return g_fail == 0 ? 0 : 1;
}

// ---------------------------------------------------------------------------
template <typename T>
bool same_bits(const std::vector<T> &a, const std::vector<T> &b) {
  return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(T)) == 0;
}

// One case through the given plan maker; the expected result is the oracle's.
template <typename T, typename Make>
void gpu_case(const std::string &name, const std::vector<uint32_t> &size,
              const std::vector<uint32_t> &perm, double alpha[2], double beta[2],
              int complex_scalars, Make make, std::mt19937_64 &rng) {
  const size_t n = prod(size);
  std::vector<T> a = random_tensor<T>(n, rng), b0 = random_tensor<T>(n, rng);
  std::vector<T> want = b0;
  const int rank = static_cast<int>(size.size());
  if (hptt_oracle_trans(Code<T>::v, rank, size.data(), perm.data(), nullptr, nullptr, alpha,
                        beta, complex_scalars, a.data(), want.data(), 1) != 0) {
    check(false, name + ": oracle");
    return;
  }
  T *da = nullptr, *db = nullptr;
  if (cudaMalloc(&da, n * sizeof(T)) != cudaSuccess ||
      cudaMalloc(&db, n * sizeof(T)) != cudaSuccess) {
    check(false, name + ": cudaMalloc");
    return;
  }
  cudaMemcpy(da, a.data(), n * sizeof(T), cudaMemcpyHostToDevice);
  cudaMemcpy(db, b0.data(), n * sizeof(T), cudaMemcpyHostToDevice);
  std::shared_ptr<hptt::trans_plan<T>> plan = make(da, db);
  check(plan != nullptr, name + ": create");
  if (plan) {
    plan->exec();
    auto ext = std::dynamic_pointer_cast<hptt::CudaTransPlan<T>>(plan);
    check(ext != nullptr, name + ": extension interface");
    if (ext) {
      check(ext->status() == 0, name + ": exec status");
      check(ext->sync() == 0, name + ": sync");
    }
    std::vector<T> got(n);
    cudaMemcpy(got.data(), db, n * sizeof(T), cudaMemcpyDeviceToHost);
    check(same_bits(got, want), name + ": result");
  }
  cudaFree(da);
  cudaFree(db);
}

template <typename T>
void gpu_type(const char *tname, std::mt19937_64 &rng) {
  using R = hptt::DeducedFloatType<T>;
  struct Shape {
    std::vector<uint32_t> size, perm;
  };
  const Shape shapes[] = {{{37, 41}, {1, 0}},
                          {{16, 9, 23}, {2, 0, 1}},
                          {{6, 7, 5, 9}, {0, 3, 2, 1}},
                          {{3, 4, 5, 6, 7}, {4, 2, 0, 3, 1}},
                          {{2, 3, 4, 5, 3, 4}, {5, 1, 3, 0, 4, 2}}};
  const double scal[][2] = {{1.0, 0.0}, {2.3, 4.2}, {-0.5, 0.0}};
  for (const Shape &s : shapes) {
    for (const auto &ab : scal) {
      double alpha[2] = {ab[0], 0.0}, beta[2] = {ab[1], 0.0};
      const std::string name = std::string(tname) + " rank " + std::to_string(s.size.size()) +
                               " a=" + std::to_string(ab[0]) + " b=" + std::to_string(ab[1]);
      gpu_case<T>(name, s.size, s.perm, alpha, beta, 0,
                  [&](T *da, T *db) {
                    return hptt::create_plan<T>(da, db, s.size, s.perm, static_cast<R>(ab[0]),
                                                static_cast<R>(ab[1]), 0);
                  },
                  rng);
    }
  }
}

// reset_data: one plan, two buffer pairs.
void gpu_reset_data(std::mt19937_64 &rng) {
  const std::vector<uint32_t> size{33, 20, 7}, perm{1, 2, 0};
  const size_t n = prod(size);
  double alpha[2] = {2.3, 0.0}, beta[2] = {4.2, 0.0};
  std::vector<float> a1 = random_tensor<float>(n, rng), a2 = random_tensor<float>(n, rng);
  std::vector<float> b = random_tensor<float>(n, rng);
  std::vector<float> w1 = b, w2 = b;
  hptt_oracle_trans(0, 3, size.data(), perm.data(), nullptr, nullptr, alpha, beta, 0,
                    a1.data(), w1.data(), 1);
  hptt_oracle_trans(0, 3, size.data(), perm.data(), nullptr, nullptr, alpha, beta, 0,
                    a2.data(), w2.data(), 1);
  float *d[4] = {nullptr, nullptr, nullptr, nullptr};
  for (auto &p : d) cudaMalloc(&p, n * sizeof(float));
  cudaMemcpy(d[0], a1.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(d[1], b.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(d[2], a2.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(d[3], b.data(), n * 4, cudaMemcpyHostToDevice);
  auto plan = hptt::create_plan<float>(d[0], d[1], size, perm, 2.3f, 4.2f, 4);
  check(plan != nullptr, "reset_data: create");
  if (plan) {
    (*plan)();
    plan->reset_data(d[2], d[3]);
    plan->set_thread_ids({0, 1, 2, 3});
    plan->exec();
    plan->unset_thread_ids();
    plan->print_plan();
    cudaDeviceSynchronize();
    std::vector<float> g1(n), g2(n);
    cudaMemcpy(g1.data(), d[1], n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(g2.data(), d[3], n * 4, cudaMemcpyDeviceToHost);
    check(same_bits(g1, w1), "reset_data: first buffers");
    check(same_bits(g2, w2), "reset_data: second buffers");
  }
  for (auto p : d) cudaFree(p);
}

// The factories, looked up by the mangled names the reference's loader uses.
template <typename T>
using Factory = hptt::CGraphTransPackBase<T> *(*)(
    const T *, T *, const hptt::TensorUInt, const std::vector<hptt::TensorUInt> &,
    const std::vector<hptt::TensorUInt> &, const hptt::DeducedFloatType<T>,
    const hptt::DeducedFloatType<T>, const hptt::TensorUInt, const double,
    const std::vector<hptt::TensorUInt> &, const std::vector<hptt::TensorUInt> &);

template <typename T>
void gpu_factory(void *lib, const char *sym, std::mt19937_64 &rng) {
  Factory<T> f = reinterpret_cast<Factory<T>>(dlsym(lib, sym));
  check(f != nullptr, std::string("dlsym ") + sym);
  if (!f) return;
  const std::vector<uint32_t> size{12, 10, 14}, perm{2, 1, 0};
  double alpha[2] = {2.3, 0.0}, beta[2] = {4.2, 0.0};
  gpu_case<T>(std::string("factory ") + sym, size, perm, alpha, beta, 0,
              [&](T *da, T *db) {
                return std::shared_ptr<hptt::trans_plan<T>>(
                    f(da, db, 3, size, perm, static_cast<hptt::DeducedFloatType<T>>(2.3),
                      static_cast<hptt::DeducedFloatType<T>>(4.2), 1, 0.0, {}, {}));
              },
              rng);
}

// C[a,b,i,j] = alpha * sum_{c,d} A[a,c,i,d] B[d,b,c,j] + beta * C through
// hptt::create_contraction, against a plain loop within the dot-product
// error bound (K + 6) u sum |a||b| + |beta c| terms.
void gpu_contraction(std::mt19937_64 &rng) {
  const uint32_t na = 6, nc = 5, ni = 7, nd = 4, nb = 9, nj = 3;
  const std::vector<uint32_t> sa{na, nc, ni, nd}, sb{nd, nb, nc, nj};
  const size_t NA = na * nc * ni * nd, NB = nd * nb * nc * nj, NC = na * nb * ni * nj;
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  std::vector<double> a(NA), b(NB), c0(NC), got(NC);
  for (auto &x : a) x = u(rng);
  for (auto &x : b) x = u(rng);
  for (auto &x : c0) x = u(rng);
  double *da = nullptr, *db = nullptr, *dc = nullptr;
  cudaMalloc(&da, NA * 8);
  cudaMalloc(&db, NB * 8);
  cudaMalloc(&dc, NC * 8);
  cudaMemcpy(da, a.data(), NA * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(db, b.data(), NB * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(dc, c0.data(), NC * 8, cudaMemcpyHostToDevice);
  const double alpha = 0.5, beta = -1.25;
  auto plan = hptt::create_contraction<double>(da, sa, {'a', 'c', 'i', 'd'}, db, sb,
                                               {'d', 'b', 'c', 'j'}, dc,
                                               {'a', 'b', 'i', 'j'}, alpha, beta);
  check(plan != nullptr, "create_contraction f64");
  if (plan) {
    check(plan->exec() == HPTT_OK && plan->exec() == HPTT_OK, "contraction exec twice");
    check(plan->sync() == HPTT_OK, "contraction sync");
    cudaMemcpy(got.data(), dc, NC * 8, cudaMemcpyDeviceToHost);
    int bad = 0;
    std::vector<double> want = c0;
    for (int rep = 0; rep < 2; ++rep) {
      std::vector<double> next(NC);
      for (uint32_t A_ = 0; A_ < na; ++A_)
        for (uint32_t B_ = 0; B_ < nb; ++B_)
          for (uint32_t I = 0; I < ni; ++I)
            for (uint32_t J = 0; J < nj; ++J) {
              double s = 0, sabs = 0;
              for (uint32_t C_ = 0; C_ < nc; ++C_)
                for (uint32_t D = 0; D < nd; ++D) {
                  const double x = a[A_ + na * (C_ + nc * (I + ni * D))];
                  const double y = b[D + nd * (B_ + nb * (C_ + nc * J))];
                  s += x * y;
                  sabs += std::fabs(x * y);
                }
              const size_t o = A_ + na * (B_ + nb * (I + ni * J));
              next[o] = alpha * s + beta * want[o];
              if (rep == 1) {
                const double tol = 2 * (nc * nd + 6) * 1.2e-16 *
                                   (std::fabs(alpha) * sabs + std::fabs(beta * want[o])) *
                                   4.0;
                if (!(std::fabs(got[o] - next[o]) <= tol + 1e-300)) ++bad;
              }
            }
      want = next;
    }
    check(bad == 0, "contraction f64 within the error bound (" + std::to_string(bad) + " bad)");
  }
  plan.reset();
  cudaFree(da);
  cudaFree(db);
  cudaFree(dc);
}

int run_gpu(const char *libpath) {
  std::mt19937_64 rng(0);
  gpu_type<float>("f32", rng);
  gpu_type<double>("f64", rng);
  gpu_type<hptt::FloatComplex>("c64", rng);
  gpu_type<hptt::DoubleComplex>("c128", rng);
  gpu_reset_data(rng);
  gpu_contraction(rng);
  {
    // complex scalars (extension)
    const std::vector<uint32_t> size{8, 6, 4, 5}, perm{3, 1, 0, 2};
    double alpha[2] = {1.5, -0.5}, beta[2] = {0.25, 1.0};
    gpu_case<hptt::FloatComplex>(
        "c64 complex scalars", size, perm, alpha, beta, 1,
        [&](hptt::FloatComplex *da, hptt::FloatComplex *db) {
          return hptt::create_plan(da, db, size, perm, std::complex<float>(1.5f, -0.5f),
                                   std::complex<float>(0.25f, 1.0f), 0);
        },
        rng);
    gpu_case<hptt::DoubleComplex>(
        "c128 complex scalars", size, perm, alpha, beta, 1,
        [&](hptt::DoubleComplex *da, hptt::DoubleComplex *db) {
          return hptt::create_plan(da, db, size, perm, std::complex<double>(1.5, -0.5),
                                   std::complex<double>(0.25, 1.0), 0);
        },
        rng);
  }
  void *lib = dlopen(libpath, RTLD_NOW | RTLD_LOCAL);
  check(lib != nullptr, std::string("dlopen ") + libpath);
  if (lib) {
    gpu_factory<float>(lib, "_Z24create_trans_plan_impl_sPKfPfjRKSt6vectorIjSaIjEES6_ffjdS6_S6_",
                       rng);
    gpu_factory<double>(lib, "_Z24create_trans_plan_impl_dPKdPdjRKSt6vectorIjSaIjEES6_ddjdS6_S6_",
                        rng);
    gpu_factory<hptt::FloatComplex>(
        lib, "_Z24create_trans_plan_impl_cPKCfPS_jRKSt6vectorIjSaIjEES7_ffjdS7_S7_", rng);
    gpu_factory<hptt::DoubleComplex>(
        lib, "_Z24create_trans_plan_impl_zPKCdPS_jRKSt6vectorIjSaIjEES7_ddjdS7_S7_", rng);
  }
  std::printf("gpu checks done, %d failure(s)\n", g_fail);
  return g_fail == 0 ? 0 : 1;
}

}  // namespace

int main(int argc, char **argv) {
  const std::string mode = argc > 1 ? argv[1] : "guard";
  if (mode == "guard") return run_guard();
  if (mode == "gpu") return run_gpu(argc > 2 ? argv[2] : "libhptt.so");
  std::printf("usage: %s guard|gpu [path/to/libhptt.so]\n", argv[0]);
  return 2;
}
