/*
 * CPU oracle: naive restatement of the reference transpose.  TEST
 * INFRASTRUCTURE ONLY (see oracle.h) -- never linked into the product.
 *
 * Indexing follows the reference's naive transpose RefTrans
 * (test/inc/hptt/test_util.tcc:143-185) generalised to outer (padded) sizes:
 *   - tensors are column-major, dimension 0 has stride 1, and stride[k+1] =
 *     outer[k] * stride[k]                     (inc/hptt/tensor.tcc:186-196)
 *   - out_size[k] = in_size[perm[k]], so output index j[k] = i[perm[k]]
 *                                   (cmake/pylib/gen_util/hptt_trans_gen.py:196-197)
 * Arithmetic follows the vector kernels (src/arch/avx2/kernel_trans_avx2.cc:68-107,
 * inc/hptt/arch/common/common_impl.h:18-33): t = fl(alpha*a); if B is updated
 * t = fl(t + fl(beta*b)); two roundings of products then one of the sum, no
 * fused multiply-add.  B is updated only when |beta| >= 1e-16
 * (inc/hptt/impl/hptt_trans_impl.h:75-78); otherwise B is never read.
 * Complex types with real scalars scale each component (inc/hptt/types.h:29-54).
 * Complex scalars (an extension the reference API cannot express) use the
 * stated order re = fl(fl(ar*xr) - fl(ai*xi)), im = fl(fl(ar*xi) + fl(ai*xr)).
 *
 * Build with -ffp-contract=off (oracle/Makefile) so that the compiler cannot
 * contract the products into FMAs.
 */
#include "oracle.h"

#include <math.h>
#include <stddef.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MAX_RANK 16

typedef struct {
  int rank;
  uint64_t size[ORACLE_MAX_RANK];     /* input extents                     */
  uint64_t sa[ORACLE_MAX_RANK];       /* input stride of input dim d       */
  uint64_t sb[ORACLE_MAX_RANK];       /* output stride of input dim d      */
} geom_t;

static int build_geom(int rank, const uint32_t *in_size, const uint32_t *perm,
                      const uint32_t *in_outer, const uint32_t *out_outer,
                      geom_t *g) {
  int seen[ORACLE_MAX_RANK] = {0};
  uint64_t out_stride[ORACLE_MAX_RANK];
  if (rank < 1 || rank > ORACLE_MAX_RANK) return -1;
  g->rank = rank;
  for (int k = 0; k < rank; ++k) {
    if (perm[k] >= (uint32_t)rank || seen[perm[k]]) return -1;
    seen[perm[k]] = 1;
    if (in_size[k] == 0) return -1;
  }
  /* input strides from input outer sizes */
  uint64_t s = 1;
  for (int d = 0; d < rank; ++d) {
    g->size[d] = in_size[d];
    g->sa[d] = s;
    uint64_t outer = in_outer ? in_outer[d] : in_size[d];
    if (outer < in_size[d]) return -1;
    s *= outer;
  }
  /* output strides from output outer sizes (indexed by output dim) */
  s = 1;
  for (int k = 0; k < rank; ++k) {
    uint64_t osz = in_size[perm[k]];
    uint64_t outer = out_outer ? out_outer[k] : osz;
    if (outer < osz) return -1;
    out_stride[k] = s;
    s *= outer;
  }
  for (int k = 0; k < rank; ++k) g->sb[perm[k]] = out_stride[k];
  return 0;
}

int hptt_oracle_update(int dtype, const double *beta, int complex_scalars) {
  if ((dtype == ORACLE_C64 || dtype == ORACLE_C128) && complex_scalars)
    return fabs(beta[0]) >= 1e-16 || fabs(beta[1]) >= 1e-16;
  if (dtype == ORACLE_F32 || dtype == ORACLE_C64)
    return fabsf((float)beta[0]) >= 1e-16;
  return fabs(beta[0]) >= 1e-16;
}

/* One element kernel per type; `o` and `i` are element offsets. */
#define DEFINE_REAL(NAME, T)                                                   \
  static void NAME(const void *in, void *out, uint64_t i, uint64_t o,          \
                   const double *al, const double *be, int upd) {              \
    const T a = ((const T *)in)[i];                                            \
    const T alpha = (T)al[0], beta = (T)be[0];                                 \
    T t = alpha * a;                                                           \
    if (upd) {                                                                 \
      T u = beta * ((T *)out)[o];                                              \
      t = t + u;                                                               \
    }                                                                          \
    ((T *)out)[o] = t;                                                         \
  }

#define DEFINE_CPLX_REAL(NAME, T)                                              \
  static void NAME(const void *in, void *out, uint64_t i, uint64_t o,          \
                   const double *al, const double *be, int upd) {              \
    const T *a = ((const T *)in) + 2 * i;                                      \
    T *b = ((T *)out) + 2 * o;                                                 \
    const T alpha = (T)al[0], beta = (T)be[0];                                 \
    T re = alpha * a[0], im = alpha * a[1];                                    \
    if (upd) {                                                                 \
      T ure = beta * b[0], uim = beta * b[1];                                  \
      re = re + ure;                                                           \
      im = im + uim;                                                           \
    }                                                                          \
    b[0] = re;                                                                 \
    b[1] = im;                                                                 \
  }

#define DEFINE_CPLX_CPLX(NAME, T)                                              \
  static void NAME(const void *in, void *out, uint64_t i, uint64_t o,          \
                   const double *al, const double *be, int upd) {              \
    const T *a = ((const T *)in) + 2 * i;                                      \
    T *b = ((T *)out) + 2 * o;                                                 \
    const T ar = (T)al[0], ai = (T)al[1], br = (T)be[0], bi = (T)be[1];        \
    T p0 = ar * a[0], p1 = ai * a[1], p2 = ar * a[1], p3 = ai * a[0];          \
    T re = p0 - p1, im = p2 + p3;                                              \
    if (upd) {                                                                 \
      T q0 = br * b[0], q1 = bi * b[1], q2 = br * b[1], q3 = bi * b[0];        \
      T ure = q0 - q1, uim = q2 + q3;                                          \
      re = re + ure;                                                           \
      im = im + uim;                                                           \
    }                                                                          \
    b[0] = re;                                                                 \
    b[1] = im;                                                                 \
  }

DEFINE_REAL(elem_f32, float)
DEFINE_REAL(elem_f64, double)
DEFINE_CPLX_REAL(elem_c64r, float)
DEFINE_CPLX_REAL(elem_c128r, double)
DEFINE_CPLX_CPLX(elem_c64c, float)
DEFINE_CPLX_CPLX(elem_c128c, double)

typedef void (*elem_fn)(const void *, void *, uint64_t, uint64_t,
                        const double *, const double *, int);

int hptt_oracle_trans(int dtype, int rank, const uint32_t *in_size,
                      const uint32_t *perm, const uint32_t *in_outer,
                      const uint32_t *out_outer, const double *alpha,
                      const double *beta, int complex_scalars,
                      const void *in, void *out, int num_threads) {
  geom_t g;
  elem_fn fn;
  if (!in_size || !perm || !alpha || !beta || !in || !out) return -1;
  if (build_geom(rank, in_size, perm, in_outer, out_outer, &g) != 0) return -1;
  switch (dtype) {
    case ORACLE_F32: fn = elem_f32; break;
    case ORACLE_F64: fn = elem_f64; break;
    case ORACLE_C64: fn = complex_scalars ? elem_c64c : elem_c64r; break;
    case ORACLE_C128: fn = complex_scalars ? elem_c128c : elem_c128r; break;
    default: return -1;
  }
  const int upd = hptt_oracle_update(dtype, beta, complex_scalars);

  /* Split the input index space into rows along input dim 0; every row is
   * independent, so rows are shared among threads. */
  uint64_t rows = 1;
  for (int d = 1; d < rank; ++d) rows *= g.size[d];
  const uint64_t n0 = g.size[0];
  if (num_threads < 1) num_threads = 1;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(num_threads)
#endif
  for (int64_t r = 0; r < (int64_t)rows; ++r) {
    uint64_t rem = (uint64_t)r, oa = 0, ob = 0;
    for (int d = 1; d < rank; ++d) {
      uint64_t c = rem % g.size[d];
      rem /= g.size[d];
      oa += c * g.sa[d];
      ob += c * g.sb[d];
    }
    for (uint64_t c0 = 0; c0 < n0; ++c0)
      fn(in, out, oa + c0, ob + c0 * g.sb[0], alpha, beta, upd);
  }
  return 0;
}
