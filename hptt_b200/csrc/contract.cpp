// Tensor contraction by transpose - GEMM - transpose (TTGT): the caller the
// transposition engine serves.  The operand transposes and the output
// transpose (which applies alpha and beta, reading C once) are this library's
// own plans; the contraction itself is one strided-batched cuBLAS GEMM.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "../../include/hptt_cuda.h"
#include "contract.h"
#include "plan.h"
#include "planner.h"

namespace hptt_b200 {

namespace {

constexpr int kMaxLabelSet = 3 * HPTT_MAX_RANK;

struct LabelSet {
  int n = 0;
  int32_t label[kMaxLabelSet];
  uint64_t ext[kMaxLabelSet];
  int find(int32_t x) const {
    for (int i = 0; i < n; ++i)
      if (label[i] == x) return i;
    return -1;
  }
  uint64_t extent(int32_t x) const {
    const int i = find(x);
    return i < 0 ? 1 : ext[i];
  }
};

int index_of(const int32_t *l, int r, int32_t x) {
  for (int i = 0; i < r; ++i)
    if (l[i] == x) return i;
  return -1;
}

// Equal label sequences once labels of extent 1 are dropped: the two
// column-major layouts then address memory identically.
bool same_layout(const int32_t *a, int na, const int32_t *b, int nb, const LabelSet &E) {
  int i = 0, j = 0;
  for (;;) {
    while (i < na && E.extent(a[i]) == 1) ++i;
    while (j < nb && E.extent(b[j]) == 1) ++j;
    if (i == na || j == nb) return i == na && j == nb;
    if (a[i] != b[j]) return false;
    ++i;
    ++j;
  }
}

// Labels of `src` that belong to class `cls` (cls[] indexed like E), in
// src's order.
int pick(const int32_t *src, int r, const int *cls, int want, const LabelSet &E, int32_t *out) {
  int n = 0;
  for (int i = 0; i < r; ++i)
    if (cls[E.find(src[i])] == want) out[n++] = src[i];
  return n;
}

int concat(int32_t *dst, const int32_t *a, int na, const int32_t *b, int nb, const int32_t *c,
           int nc) {
  int n = 0;
  for (int i = 0; i < na; ++i) dst[n++] = a[i];
  for (int i = 0; i < nb; ++i) dst[n++] = b[i];
  for (int i = 0; i < nc; ++i) dst[n++] = c[i];
  return n;
}

uint64_t align256(uint64_t x) { return (x + 255) & ~uint64_t(255); }

}  // namespace

int contract_analyze(int dtype, int ra, const uint32_t *sa, const int32_t *la, int rb,
                     const uint32_t *sb, const int32_t *lb, int rc, const int32_t *lc,
                     ContractLayout *out) {
  const int es = elem_bytes(dtype);
  if (es == 0) return ST_BAD_DTYPE;
  if (ra < 1 || ra > HPTT_MAX_RANK || rb < 1 || rb > HPTT_MAX_RANK || rc < 0 ||
      rc > HPTT_MAX_RANK)
    return ST_BAD_RANK;
  if (!sa || !la || !sb || !lb || (rc > 0 && !lc)) return ST_BAD_SIZE_VECTOR;
  ContractLayout L;
  L.dtype = dtype;
  L.ra = ra;
  L.rb = rb;
  L.rc = rc;
  LabelSet E;
  // labels unique per tensor; a label shared by A and B has one extent
  for (int t = 0; t < 2; ++t) {
    const int r = t ? rb : ra;
    const uint32_t *s = t ? sb : sa;
    const int32_t *l = t ? lb : la;
    for (int i = 0; i < r; ++i) {
      if (s[i] == 0) return ST_BAD_SIZE_VALUE;
      if (index_of(l, i, l[i]) >= 0) return ST_LABELS;
      const int f = E.find(l[i]);
      if (f >= 0) {
        if (E.ext[f] != s[i]) return ST_LABELS;
      } else {
        E.label[E.n] = l[i];
        E.ext[E.n] = s[i];
        ++E.n;
      }
      (t ? L.lb : L.la)[i] = l[i];
      (t ? L.sb : L.sa)[i] = s[i];
    }
  }
  for (int i = 0; i < rc; ++i) {
    if (index_of(lc, i, lc[i]) >= 0 || E.find(lc[i]) < 0) return ST_LABELS;
    L.lc[i] = lc[i];
    L.sc[i] = static_cast<uint32_t>(E.extent(lc[i]));
  }
  // classes: 0 M (A, C), 1 N (B, C), 2 K (A, B), 3 BATCH (A, B, C)
  int cls[kMaxLabelSet];
  for (int i = 0; i < E.n; ++i) {
    const bool inA = index_of(la, ra, E.label[i]) >= 0;
    const bool inB = index_of(lb, rb, E.label[i]) >= 0;
    const bool inC = index_of(lc, rc, E.label[i]) >= 0;
    if (inA && inB)
      cls[i] = inC ? 3 : 2;
    else if (!inC)
      return ST_LABELS;  // summed over one operand only: not a GEMM
    else
      cls[i] = inA ? 0 : 1;
  }
  auto prod = [&](const int32_t *l, int n, uint64_t *v) {
    uint64_t p = 1;
    for (int i = 0; i < n; ++i) {
      const uint64_t e = E.extent(l[i]);
      if (p > (uint64_t(1) << 62) / e) return false;
      p *= e;
    }
    *v = p;
    return true;
  };

  // candidate orders of each class
  int32_t mo[2][HPTT_MAX_RANK], no[2][HPTT_MAX_RANK], ko[2][HPTT_MAX_RANK],
      bo[3][HPTT_MAX_RANK];
  const int nm = pick(lc, rc, cls, 0, E, mo[0]);
  pick(la, ra, cls, 0, E, mo[1]);
  const int nn = pick(lc, rc, cls, 1, E, no[0]);
  pick(lb, rb, cls, 1, E, no[1]);
  const int nk = pick(la, ra, cls, 2, E, ko[0]);
  pick(lb, rb, cls, 2, E, ko[1]);
  const int nb = pick(lc, rc, cls, 3, E, bo[0]);
  pick(la, ra, cls, 3, E, bo[1]);
  pick(lb, rb, cls, 3, E, bo[2]);

  if (!prod(la, ra, &L.elems_a) || !prod(lb, rb, &L.elems_b) || !prod(lc, rc, &L.elems_c) ||
      !prod(mo[0], nm, &L.m) || !prod(no[0], nn, &L.n) || !prod(ko[0], nk, &L.k) ||
      !prod(bo[0], nb, &L.batch))
    return ST_TOO_LARGE;
  const uint64_t imax = 0x7fffffffull;
  if (L.m > imax || L.n > imax || L.k > imax || L.batch > imax) return ST_TOO_LARGE;

  // Fewest transposed elements wins; ties keep the earliest candidate
  // (output-side orders, A-hat [M, K], B-hat [K, N], no swap).
  uint64_t best = ~uint64_t(0);
  for (int swap = 0; swap < 2; ++swap)
    for (int akm = 0; akm < 2; ++akm)
      for (int bnk = 0; bnk < 2; ++bnk)
        for (int im = 0; im < 2; ++im)
          for (int in = 0; in < 2; ++in)
            for (int ik = 0; ik < 2; ++ik)
              for (int ib = 0; ib < 3; ++ib) {
                int32_t ah[HPTT_MAX_RANK], bh[HPTT_MAX_RANK], ch[HPTT_MAX_RANK];
                if (akm)
                  concat(ah, ko[ik], nk, mo[im], nm, bo[ib], nb);
                else
                  concat(ah, mo[im], nm, ko[ik], nk, bo[ib], nb);
                if (bnk)
                  concat(bh, no[in], nn, ko[ik], nk, bo[ib], nb);
                else
                  concat(bh, ko[ik], nk, no[in], nn, bo[ib], nb);
                if (swap)
                  concat(ch, no[in], nn, mo[im], nm, bo[ib], nb);
                else
                  concat(ch, mo[im], nm, no[in], nn, bo[ib], nb);
                const int ta = !same_layout(la, ra, ah, ra, E);
                const int tb = !same_layout(lb, rb, bh, rb, E);
                const int tc = !same_layout(lc, rc, ch, rc, E);
                const uint64_t cost = ta * L.elems_a + tb * L.elems_b + tc * L.elems_c;
                if (cost >= best) continue;
                best = cost;
                L.swap = swap;
                L.a_km = akm;
                L.b_nk = bnk;
                L.tr_a = ta;
                L.tr_b = tb;
                L.tr_c = tc;
                L.nm = nm;
                L.nn = nn;
                L.nk = nk;
                L.nbat = nb;
                std::memcpy(L.ml, mo[im], sizeof(int32_t) * nm);
                std::memcpy(L.nl, no[in], sizeof(int32_t) * nn);
                std::memcpy(L.kl, ko[ik], sizeof(int32_t) * nk);
                std::memcpy(L.bl, bo[ib], sizeof(int32_t) * nb);
                for (int i = 0; i < ra; ++i)
                  L.pa_perm[i] = static_cast<uint32_t>(index_of(la, ra, ah[i]));
                for (int i = 0; i < rb; ++i)
                  L.pb_perm[i] = static_cast<uint32_t>(index_of(lb, rb, bh[i]));
                for (int i = 0; i < rc; ++i) {
                  L.chat_size[i] = static_cast<uint32_t>(E.extent(ch[i]));
                  L.pc_perm[i] = static_cast<uint32_t>(index_of(ch, rc, lc[i]));
                }
              }

  uint64_t off = 0;
  if (L.tr_a) {
    L.off_a = off;
    off = align256(off + L.elems_a * es);
  }
  if (L.tr_b) {
    L.off_b = off;
    off = align256(off + L.elems_b * es);
  }
  if (L.tr_c) {
    L.off_c = off;
    off = align256(off + L.elems_c * es);
  }
  L.off_blas = off;
  L.ws_bytes = off + kBlasWorkspaceBytes;
  L.moved_bytes = 2ull * es * (L.tr_a * L.elems_a + L.tr_b * L.elems_b + L.tr_c * L.elems_c);
  *out = L;
  return ST_OK;
}

void contract_describe(const ContractLayout &L, char *buf, size_t len) {
  auto labels = [](const int32_t *l, int n) {
    std::string s = "[";
    for (int i = 0; i < n; ++i) {
      if (i) s += ",";
      s += std::to_string(l[i]);
    }
    return s + "]";
  };
  const char *dt[] = {"f32", "f64", "c64", "c128"};
  std::string s = "hptt-b200 contraction (transpose - GEMM - transpose)\n";
  s += std::string("  dtype ") + dt[L.dtype & 3] + ", M " + labels(L.ml, L.nm) + " = " +
       std::to_string(L.m) + ", N " + labels(L.nl, L.nn) + " = " + std::to_string(L.n) +
       ", K " + labels(L.kl, L.nk) + " = " + std::to_string(L.k) + ", batch " +
       labels(L.bl, L.nbat) + " = " + std::to_string(L.batch) + "\n";
  s += std::string("  A-hat ") + (L.a_km ? "[K,M]" : "[M,K]") +
       (L.tr_a ? " (transposed)" : " (A in place)") + ", B-hat " + (L.b_nk ? "[N,K]" : "[K,N]") +
       (L.tr_b ? " (transposed)" : " (B in place)") + "\n";
  s += std::string("  GEMM writes ") + (L.swap ? "[N,M]" : "[M,N]") +
       (L.tr_c ? " to C-hat, output transpose applies alpha, beta"
               : " into C with alpha, beta") +
       "\n";
  s += "  workspace " + std::to_string(L.ws_bytes) + " bytes, transposes move " +
       std::to_string(L.moved_bytes) + " bytes\n";
  if (buf && len) {
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = 0;
  }
}

namespace {

constexpr uint32_t kContractMagic = 0x54544754u;  // "TTGT"

struct Contraction {
  uint32_t magic = kContractMagic;
  ContractLayout L;
  const void *A = nullptr, *B = nullptr;
  void *C = nullptr;
  double alpha[2] = {1.0, 0.0}, beta[2] = {0.0, 0.0};
  int complex_scalars = 0;
  bool update = false;
  hptt_cuda_plan_t ta = nullptr, tb = nullptr, tc = nullptr;
  unsigned char *ws = nullptr;
  bool own_ws = false;
  cublasHandle_t blas = nullptr;
  cudaStream_t stream = nullptr;           // stream of hptt_cuda_contract_exec
  cudaStream_t cap = nullptr, side = nullptr;  // capture streams
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int use_graph = 1;
  int execs = 0;  // the first exec runs directly (loads every kernel), later ones replay
};

bool valid(const Contraction *c) { return c && c->magic == kContractMagic; }

void drop_graph(Contraction *c) {
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  c->gexec = nullptr;
  c->graph = nullptr;
}

// B is read by the output step when |beta| >= 1e-16, the transpose plans' rule.
bool beta_reads(int dtype, const double *beta, int complex_scalars) {
  HpttArgs a{};
  a.p.dtype = dtype;
  const double one[2] = {1.0, 0.0};
  set_scalars(&a, one, beta, complex_scalars);
  return a.update != 0;
}

int gemm(Contraction *c, cudaStream_t s) {
  const ContractLayout &L = c->L;
  const void *ah = L.tr_a ? static_cast<const void *>(c->ws + L.off_a) : c->A;
  const void *bh = L.tr_b ? static_cast<const void *>(c->ws + L.off_b) : c->B;
  void *ch = L.tr_c ? static_cast<void *>(c->ws + L.off_c) : c->C;
  const int m = static_cast<int>(L.m), n = static_cast<int>(L.n), k = static_cast<int>(L.k);
  const long long sa = static_cast<long long>(L.m * L.k);
  const long long sb = static_cast<long long>(L.k * L.n);
  const long long scs = static_cast<long long>(L.m * L.n);
  int M, N, ldx, ldy;
  long long sx, sy;
  cublasOperation_t ox, oy;
  const void *X, *Y;
  if (!L.swap) {  // C-hat[m,n] = op(A-hat) op(B-hat)
    M = m;
    N = n;
    X = ah;
    ox = L.a_km ? CUBLAS_OP_T : CUBLAS_OP_N;
    ldx = L.a_km ? k : m;
    sx = sa;
    Y = bh;
    oy = L.b_nk ? CUBLAS_OP_T : CUBLAS_OP_N;
    ldy = L.b_nk ? n : k;
    sy = sb;
  } else {  // C-hat[n,m] = B-hat^T A-hat^T
    M = n;
    N = m;
    X = bh;
    ox = L.b_nk ? CUBLAS_OP_N : CUBLAS_OP_T;
    ldx = L.b_nk ? n : k;
    sx = sb;
    Y = ah;
    oy = L.a_km ? CUBLAS_OP_N : CUBLAS_OP_T;
    ldy = L.a_km ? k : m;
    sy = sa;
  }
  // scalars: applied by the GEMM only when no output transpose follows
  double al[2] = {1.0, 0.0}, be[2] = {0.0, 0.0};
  if (!L.tr_c) {
    al[0] = c->alpha[0];
    al[1] = c->complex_scalars ? c->alpha[1] : 0.0;
    if (c->update) {
      be[0] = c->beta[0];
      be[1] = c->complex_scalars ? c->beta[1] : 0.0;
    }
  }
  const int batch = static_cast<int>(L.batch);
  if (cublasSetStream(c->blas, s) != CUBLAS_STATUS_SUCCESS) return ST_BLAS;
  cublasStatus_t st;
  switch (L.dtype) {
    case DT_F32: {
      const float a = static_cast<float>(al[0]), b = static_cast<float>(be[0]);
      st = cublasSgemmStridedBatched(c->blas, ox, oy, M, N, k, &a, static_cast<const float *>(X),
                                     ldx, sx, static_cast<const float *>(Y), ldy, sy, &b,
                                     static_cast<float *>(ch), M, scs, batch);
      break;
    }
    case DT_F64:
      st = cublasDgemmStridedBatched(c->blas, ox, oy, M, N, k, &al[0],
                                     static_cast<const double *>(X), ldx, sx,
                                     static_cast<const double *>(Y), ldy, sy, &be[0],
                                     static_cast<double *>(ch), M, scs, batch);
      break;
    case DT_C64: {
      const cuComplex a = make_cuComplex(static_cast<float>(al[0]), static_cast<float>(al[1]));
      const cuComplex b = make_cuComplex(static_cast<float>(be[0]), static_cast<float>(be[1]));
      st = cublasCgemmStridedBatched(c->blas, ox, oy, M, N, k, &a,
                                     static_cast<const cuComplex *>(X), ldx, sx,
                                     static_cast<const cuComplex *>(Y), ldy, sy, &b,
                                     static_cast<cuComplex *>(ch), M, scs, batch);
      break;
    }
    default: {
      const cuDoubleComplex a = make_cuDoubleComplex(al[0], al[1]);
      const cuDoubleComplex b = make_cuDoubleComplex(be[0], be[1]);
      st = cublasZgemmStridedBatched(c->blas, ox, oy, M, N, k, &a,
                                     static_cast<const cuDoubleComplex *>(X), ldx, sx,
                                     static_cast<const cuDoubleComplex *>(Y), ldy, sy, &b,
                                     static_cast<cuDoubleComplex *>(ch), M, scs, batch);
      break;
    }
  }
  return st == CUBLAS_STATUS_SUCCESS ? ST_OK : ST_BLAS;
}

// Enqueue the whole contraction on `s`; with `side` set, the B transpose runs
// there, joined back before the GEMM.
int enqueue(Contraction *c, cudaStream_t s, cudaStream_t side) {
  int st;
  if (side && c->ta && c->tb) {
    if (cudaEventRecord(c->fork, s) != cudaSuccess ||
        cudaStreamWaitEvent(side, c->fork, 0) != cudaSuccess)
      return ST_CUDA;
    if ((st = hptt_cuda_plan_exec_on(c->tb, side)) != ST_OK) return st;
    if (cudaEventRecord(c->join, side) != cudaSuccess) return ST_CUDA;
    if ((st = hptt_cuda_plan_exec_on(c->ta, s)) != ST_OK) return st;
    if (cudaStreamWaitEvent(s, c->join, 0) != cudaSuccess) return ST_CUDA;
  } else {
    if (c->ta && (st = hptt_cuda_plan_exec_on(c->ta, s)) != ST_OK) return st;
    if (c->tb && (st = hptt_cuda_plan_exec_on(c->tb, s)) != ST_OK) return st;
  }
  if ((st = gemm(c, s)) != ST_OK) return st;
  if (c->tc && (st = hptt_cuda_plan_exec_on(c->tc, s)) != ST_OK) return st;
  return ST_OK;
}

// Capture the contraction once into a graph (transposes of A and B as
// parallel branches).  On any capture failure the contraction keeps running
// its direct form.
void capture(Contraction *c) {
  if (cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    c->use_graph = 0;
    return;
  }
  const int st = enqueue(c, c->cap, c->side);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->cap, &g);
  if (st != ST_OK || e != cudaSuccess || !g ||
      cudaGraphInstantiate(&c->gexec, g, 0) != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    c->gexec = nullptr;
    cudaGetLastError();
    c->use_graph = 0;
    return;
  }
  c->graph = g;
}

int exec_on(Contraction *c, cudaStream_t s) {
  if (!c->A || !c->B || !c->C) return ST_NULL_DATA;
  if (c->use_graph && c->execs > 0 && !c->gexec) capture(c);
  ++c->execs;
  if (c->use_graph && c->gexec)
    return cudaGraphLaunch(c->gexec, s) == cudaSuccess ? ST_OK : ST_CUDA;
  return enqueue(c, s, nullptr);
}

void destroy(Contraction *c) {
  drop_graph(c);
  if (c->ta) hptt_cuda_plan_destroy(c->ta);
  if (c->tb) hptt_cuda_plan_destroy(c->tb);
  if (c->tc) hptt_cuda_plan_destroy(c->tc);
  if (c->blas) cublasDestroy(c->blas);
  if (c->fork) cudaEventDestroy(c->fork);
  if (c->join) cudaEventDestroy(c->join);
  if (c->cap) cudaStreamDestroy(c->cap);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->own_ws && c->ws) cudaFree(c->ws);
  c->magic = 0;
  delete c;
}

}  // namespace
}  // namespace hptt_b200

using namespace hptt_b200;

extern "C" {

int hptt_cuda_contract_inspect(int dtype, uint32_t rank_a, const uint32_t *size_a,
                               const int32_t *labels_a, uint32_t rank_b,
                               const uint32_t *size_b, const int32_t *labels_b,
                               uint32_t rank_c, const int32_t *labels_c, char *buf, size_t len,
                               uint64_t *workspace_bytes) {
  ContractLayout L;
  const int st = contract_analyze(dtype, static_cast<int>(rank_a), size_a, labels_a,
                                  static_cast<int>(rank_b), size_b, labels_b,
                                  static_cast<int>(rank_c), labels_c, &L);
  if (st != ST_OK) return st;
  contract_describe(L, buf, len);
  if (workspace_bytes) *workspace_bytes = L.ws_bytes;
  return HPTT_OK;
}

int hptt_cuda_contract_create(int dtype, uint32_t rank_a, const uint32_t *size_a,
                              const int32_t *labels_a, uint32_t rank_b, const uint32_t *size_b,
                              const int32_t *labels_b, uint32_t rank_c,
                              const int32_t *labels_c, const double *alpha,
                              const double *beta, int complex_scalars, const void *A,
                              const void *B, void *C, void *workspace,
                              uint64_t workspace_bytes, hptt_cuda_contract_t *out) {
  if (!out) return HPTT_ERR_HANDLE;
  *out = nullptr;
  if (!A || !B || !C) return HPTT_ERR_NULL_DATA;
  if (!alpha || !beta) return HPTT_ERR_SIZE_VALUE;
  Contraction *c = new (std::nothrow) Contraction();
  if (!c) return HPTT_ERR_ALLOC;
  int st = contract_analyze(dtype, static_cast<int>(rank_a), size_a, labels_a,
                            static_cast<int>(rank_b), size_b, labels_b,
                            static_cast<int>(rank_c), labels_c, &c->L);
  if (st != ST_OK) {
    delete c;
    return st;
  }
  const ContractLayout &L = c->L;
  const bool cplx = dtype == DT_C64 || dtype == DT_C128;
  c->A = A;
  c->B = B;
  c->C = C;
  c->complex_scalars = cplx && complex_scalars;
  c->alpha[0] = alpha[0];
  c->alpha[1] = c->complex_scalars ? alpha[1] : 0.0;
  c->beta[0] = beta[0];
  c->beta[1] = c->complex_scalars ? beta[1] : 0.0;
  c->update = beta_reads(dtype, c->beta, c->complex_scalars);
  if (L.tr_c && c->update) c->L.moved_bytes += L.elems_c * elem_bytes(dtype);

  if (workspace) {
    if (workspace_bytes < L.ws_bytes || (reinterpret_cast<uintptr_t>(workspace) & 255)) {
      delete c;
      return HPTT_ERR_BUDGET;
    }
    c->ws = static_cast<unsigned char *>(workspace);
  } else {
    if (cudaMalloc(reinterpret_cast<void **>(&c->ws), L.ws_bytes) != cudaSuccess) {
      cudaGetLastError();
      delete c;
      return HPTT_ERR_ALLOC;
    }
    c->own_ws = true;
  }
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  if (L.tr_a)
    st = hptt_cuda_plan_create(dtype, L.ra, L.sa, L.pa_perm, nullptr, nullptr, one, zero, 0, A,
                               c->ws + L.off_a, 0, 0.0, &c->ta);
  if (st == ST_OK && L.tr_b)
    st = hptt_cuda_plan_create(dtype, L.rb, L.sb, L.pb_perm, nullptr, nullptr, one, zero, 0, B,
                               c->ws + L.off_b, 0, 0.0, &c->tb);
  if (st == ST_OK && L.tr_c)
    st = hptt_cuda_plan_create(dtype, L.rc, L.chat_size, L.pc_perm, nullptr, nullptr, c->alpha,
                               c->beta, c->complex_scalars, c->ws + L.off_c, C, 0, 0.0, &c->tc);
  if (st == ST_OK) {
    if (cublasCreate(&c->blas) != CUBLAS_STATUS_SUCCESS ||
        cublasSetWorkspace(c->blas, c->ws + L.off_blas, kBlasWorkspaceBytes) !=
            CUBLAS_STATUS_SUCCESS ||
        cublasSetMathMode(c->blas, CUBLAS_DEFAULT_MATH) != CUBLAS_STATUS_SUCCESS)
      st = ST_BLAS;
  }
  if (st == ST_OK &&
      (cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking) != cudaSuccess ||
       cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
       cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) != cudaSuccess ||
       cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming) != cudaSuccess))
    st = ST_CUDA;
  if (st != ST_OK) {
    cudaGetLastError();
    destroy(c);
    return st;
  }
  *out = reinterpret_cast<hptt_cuda_contract_t>(c);
  return HPTT_OK;
}

int hptt_cuda_contract_exec(hptt_cuda_contract_t plan) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  return exec_on(c, c->stream);
}

int hptt_cuda_contract_exec_on(hptt_cuda_contract_t plan, void *stream) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  return exec_on(c, static_cast<cudaStream_t>(stream));
}

int hptt_cuda_contract_reset_data(hptt_cuda_contract_t plan, const void *A, const void *B,
                                  void *C) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  c->A = A;
  c->B = B;
  c->C = C;
  if (c->ta) hptt_cuda_plan_reset_data(c->ta, A, c->ws + c->L.off_a);
  if (c->tb) hptt_cuda_plan_reset_data(c->tb, B, c->ws + c->L.off_b);
  if (c->tc) hptt_cuda_plan_reset_data(c->tc, c->ws + c->L.off_c, C);
  drop_graph(c);
  return HPTT_OK;
}

int hptt_cuda_contract_set_coef(hptt_cuda_contract_t plan, const double *alpha,
                                const double *beta, int complex_scalars) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  if (!alpha || !beta) return HPTT_ERR_SIZE_VALUE;
  const int dt = c->L.dtype;
  const bool cplx = dt == DT_C64 || dt == DT_C128;
  c->complex_scalars = cplx && complex_scalars;
  c->alpha[0] = alpha[0];
  c->alpha[1] = c->complex_scalars ? alpha[1] : 0.0;
  c->beta[0] = beta[0];
  c->beta[1] = c->complex_scalars ? beta[1] : 0.0;
  const bool was = c->update;
  c->update = beta_reads(dt, c->beta, c->complex_scalars);
  if (c->L.tr_c) {
    const uint64_t cb = c->L.elems_c * elem_bytes(dt);
    if (was && !c->update) c->L.moved_bytes -= cb;
    if (!was && c->update) c->L.moved_bytes += cb;
    const int st = hptt_cuda_plan_set_coef(c->tc, c->alpha, c->beta, c->complex_scalars);
    if (st != HPTT_OK) return st;
  }
  drop_graph(c);
  return HPTT_OK;
}

int hptt_cuda_contract_set_stream(hptt_cuda_contract_t plan, void *stream) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  c->stream = static_cast<cudaStream_t>(stream);
  return HPTT_OK;
}

int hptt_cuda_contract_set_graph(hptt_cuda_contract_t plan, int use_graph) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  c->use_graph = use_graph ? 1 : 0;
  drop_graph(c);
  return HPTT_OK;
}

int hptt_cuda_contract_sync(hptt_cuda_contract_t plan) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  return cudaStreamSynchronize(c->stream) == cudaSuccess ? HPTT_OK : HPTT_ERR_CUDA;
}

int hptt_cuda_contract_info(hptt_cuda_contract_t plan, hptt_cuda_contract_stats *info) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  if (!info) return HPTT_ERR_SIZE_VALUE;
  const ContractLayout &L = c->L;
  const bool cplx = L.dtype == DT_C64 || L.dtype == DT_C128;
  std::memset(info, 0, sizeof(*info));
  info->m = L.m;
  info->n = L.n;
  info->k = L.k;
  info->batch = L.batch;
  info->flops = (cplx ? 8ull : 2ull) * L.m * L.n * L.k * L.batch;
  info->transpose_bytes = L.moved_bytes;
  info->workspace_bytes = L.ws_bytes;
  info->transposes = static_cast<uint32_t>(L.tr_a + L.tr_b + L.tr_c);
  info->graph = c->gexec ? 1u : 0u;
  return HPTT_OK;
}

int hptt_cuda_contract_describe(hptt_cuda_contract_t plan, char *buf, size_t len) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  if (!buf || !len) return HPTT_ERR_SIZE_VALUE;
  contract_describe(c->L, buf, len);
  const size_t used = std::strlen(buf);
  if (used + 1 < len)
    std::snprintf(buf + used, len - used, "  launch: %s\n",
                  !c->use_graph ? "direct" : (c->gexec ? "graph" : "direct, graph on next exec"));
  return HPTT_OK;
}

int hptt_cuda_contract_destroy(hptt_cuda_contract_t plan) {
  Contraction *c = reinterpret_cast<Contraction *>(plan);
  if (!valid(c)) return HPTT_ERR_HANDLE;
  destroy(c);
  return HPTT_OK;
}

}  // extern "C"
