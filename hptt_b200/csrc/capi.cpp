// C ABI of libhptt_cuda.so: single-transpose plans.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/hptt_cuda.h"
#include "autotune.h"
#include "launch.h"
#include "plan.h"
#include "planner.h"
#include "tables.h"

namespace hptt_b200 {

bool plan_valid(const Plan *p) { return p && p->magic == kPlanMagic; }

void set_scalars(HpttArgs *a, const double *alpha, const double *beta,
                 int complex_scalars) {
  const bool cplx_type = a->p.dtype == DT_C64 || a->p.dtype == DT_C128;
  const bool use_cplx = cplx_type && complex_scalars;
  a->alpha[0] = alpha[0];
  a->alpha[1] = use_cplx ? alpha[1] : 0.0;
  a->beta[0] = beta[0];
  a->beta[1] = use_cplx ? beta[1] : 0.0;
  // Update rule: |beta| >= 1e-16 (inc/hptt/impl/hptt_trans_impl.h:75-78), on
  // the scalar in the element's precision.
  bool upd;
  if (use_cplx) {
    upd = std::fabs(a->beta[0]) >= 1e-16 || std::fabs(a->beta[1]) >= 1e-16;
  } else if (a->p.dtype == DT_F32 || a->p.dtype == DT_C64) {
    upd = std::fabs(static_cast<float>(a->beta[0])) >= 1e-16;
  } else {
    upd = std::fabs(a->beta[0]) >= 1e-16;
  }
  a->update = upd ? 1 : 0;
  // A bit copy equals fl(1 * a) per component for real scalars only.  With
  // complex scalars alpha = 1+0i still computes fl(fl(1*xr) - fl(0*xi)) and
  // fl(fl(1*xi) + fl(0*xr)): -0 parts can turn +0, and an infinite or NaN
  // part makes the other part NaN, so that mode never takes the copy.
  const bool alpha_one = !use_cplx && ((a->p.dtype == DT_F32 || a->p.dtype == DT_C64)
                                           ? static_cast<float>(a->alpha[0]) == 1.0f
                                           : a->alpha[0] == 1.0);
  if (!upd && alpha_one)
    a->mode = MODE_COPY;
  else
    a->mode = use_cplx ? MODE_CPLX : MODE_REAL;
}

int plan_tiles(Plan *p, const TileParams &params) {
  p->params = params;
  int st = choose_tile(p->args.p, params, p->args.update, &p->args.t);
  if (st != ST_OK) return st;
  p->vec = p->args.t.kind == KIND_ROWS ? p->args.t.vec : 1;
  if (p->args.t.kind == KIND_TTILE) {
    // pointers off a 16-byte boundary (no tensor map) take the element tile
    TileParams sp = params;
    sp.tt = 0;
    sp.vt = 0;
    st = choose_tile(p->args.p, sp, p->args.update, &p->tile_scalar);
    if (st != ST_OK) return st;
  } else if (p->args.t.kind == KIND_ROWS && p->vec > 1) {
    // same problem without vector accesses, for pointers that are not
    // aligned to the planned vector
    TileParams sp = params;
    sp.max_vec_bytes = elem_bytes(p->args.p.dtype);
    st = choose_tile(p->args.p, sp, p->args.update, &p->tile_scalar);
    if (st != ST_OK) return st;
  } else {
    p->tile_scalar = p->args.t;
  }
  // device offset tables (a few KB, read through L1 by every CTA)
  plan_free_tables(p);
  auto upload = [](const HpttProblem &prob, const HpttTile &t, void **dst) -> int {
    std::vector<unsigned char> host;
    build_tables(prob, t, &host);
    if (cudaMalloc(dst, host.size()) != cudaSuccess) {
      cudaGetLastError();
      *dst = nullptr;
      return ST_ALLOC;
    }
    if (cudaMemcpy(*dst, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return ST_CUDA;
    return ST_OK;
  };
  st = upload(p->args.p, p->args.t, &p->dtab);
  if (st != ST_OK) return st;
  if ((p->args.t.kind == KIND_ROWS && p->vec > 1) || p->args.t.kind == KIND_TTILE) {
    st = upload(p->args.p, p->tile_scalar, &p->dtab_scalar);
    if (st != ST_OK) return st;
  } else {
    p->dtab_scalar = p->dtab;
  }
  if (p->args.t.nt != kBatchThreads || p->args.t.kind == KIND_VTILE ||
      p->args.t.kind == KIND_TTILE) {
    // the batch kernels run the 256-thread tile and rows forms only
    TileParams bp = params;
    bp.nt = kBatchThreads;
    bp.vt = 0;
    bp.tt = 0;
    bp.max_vec_bytes = elem_bytes(p->args.p.dtype);  // rows: the scalar form
    st = choose_tile(p->args.p, bp, p->args.update, &p->tile_batch);
    if (st != ST_OK) return st;
    st = upload(p->args.p, p->tile_batch, &p->dtab_batch);
    if (st != ST_OK) return st;
  } else {
    p->tile_batch = p->args.t;
    p->dtab_batch = p->dtab;
  }
  // grid: resident CTAs on every SM, capped by the tile count
  auto size_grid = [&](const HpttTile &t, int vec, int *grid) -> int {
    HpttArgs a = p->args;
    a.t = t;
    int per_sm = 0;
    if (occupancy(a, vec, &per_sm) != cudaSuccess || per_sm < 1) return ST_CUDA;
    if (params.ctas_per_sm > 0 && params.ctas_per_sm < per_sm) per_sm = params.ctas_per_sm;
    int64_t g = static_cast<int64_t>(per_sm) * p->sm_count;
    if (g > t.num_tiles) g = t.num_tiles;
    if (g < 1) g = 1;
    *grid = static_cast<int>(g);
    return ST_OK;
  };
  st = size_grid(p->args.t, p->vec, &p->grid);
  if (st != ST_OK) return st;
  return size_grid(p->tile_scalar, 1, &p->grid_scalar);
}

int plan_vec_for_ptrs(const Plan *p) {
  if (p->vec <= 1) return 1;
  const uintptr_t bytes = static_cast<uintptr_t>(p->vec) * elem_bytes(p->args.p.dtype);
  const uintptr_t a = reinterpret_cast<uintptr_t>(p->args.A);
  const uintptr_t b = reinterpret_cast<uintptr_t>(p->args.B);
  return (a % bytes == 0 && b % bytes == 0) ? p->vec : 1;
}

int plan_enqueue_with(const Plan *p, const void *A, void *B, cudaStream_t stream) {
  if (!A || !B) return ST_NULL_DATA;
  HpttArgs a = p->args;
  a.A = A;
  a.B = B;
  int vec = p->vec;
  if (vec > 1) {
    const uintptr_t vb = static_cast<uintptr_t>(vec) * elem_bytes(a.p.dtype);
    if (reinterpret_cast<uintptr_t>(A) % vb || reinterpret_cast<uintptr_t>(B) % vb) vec = 1;
  }
  if (a.t.kind == KIND_TTILE &&
      ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)) {
    // no tensor map for this base: the plan's element tile
    a.t = p->tile_scalar;
    a.tables = p->dtab_scalar;
    const cudaError_t e2 = launch_single(a, 1, p->grid_scalar, stream);
    return e2 == cudaSuccess ? ST_OK : ST_CUDA;
  }
  cudaError_t e;
  if (vec == p->vec) {
    a.tables = p->dtab;
    e = launch_single(a, vec, p->grid, stream);
  } else {
    a.t = p->tile_scalar;
    a.tables = p->dtab_scalar;
    e = launch_single(a, 1, p->grid_scalar, stream);
  }
  return e == cudaSuccess ? ST_OK : ST_CUDA;
}

int plan_enqueue(Plan *p, cudaStream_t stream) {
  return plan_enqueue_with(p, p->args.A, p->args.B, stream);
}

void plan_free_tables(Plan *p) {
  if (p->dtab_scalar && p->dtab_scalar != p->dtab) cudaFree(p->dtab_scalar);
  if (p->dtab_batch && p->dtab_batch != p->dtab) cudaFree(p->dtab_batch);
  if (p->dtab) cudaFree(p->dtab);
  p->dtab = nullptr;
  p->dtab_scalar = nullptr;
  p->dtab_batch = nullptr;
}

}  // namespace hptt_b200

using namespace hptt_b200;

extern "C" {

int hptt_cuda_plan_create(int dtype, uint32_t rank, const uint32_t *in_size,
                          const uint32_t *perm, const uint32_t *in_outer,
                          const uint32_t *out_outer, const double *alpha,
                          const double *beta, int complex_scalars,
                          const void *in, void *out, uint32_t num_threads,
                          double tuning_timeout, hptt_cuda_plan_t *plan) {
  (void)num_threads;
  if (!plan) return HPTT_ERR_HANDLE;
  *plan = nullptr;
  // argument guard in the reference's order (src/hptt.cc:25-56)
  if (!in || !out) return HPTT_ERR_NULL_DATA;
  if (elem_bytes(dtype) == 0) return HPTT_ERR_DTYPE;
  int st = validate(static_cast<int>(rank), in_size, perm, in_outer, out_outer,
                    in_outer ? static_cast<int>(rank) : 0,
                    out_outer ? static_cast<int>(rank) : 0);
  if (st != ST_OK) return st;
  if (!alpha || !beta) return HPTT_ERR_SIZE_VALUE;

  Plan *p = new (std::nothrow) Plan();
  if (!p) return HPTT_ERR_ALLOC;
  st = fuse(dtype, static_cast<int>(rank), in_size, perm, in_outer, out_outer, &p->args.p);
  if (st != ST_OK) {
    delete p;
    return st;
  }
  p->elements = 1;
  for (uint32_t d = 0; d < rank; ++d) p->elements *= in_size[d];
  p->args.A = in;
  p->args.B = out;
  set_scalars(&p->args, alpha, beta, complex_scalars);
  if (cudaGetDevice(&p->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, p->device) !=
          cudaSuccess) {
    delete p;
    return HPTT_ERR_NO_DEVICE;
  }
  TileParams params;
  bool have = false;
  if (tuning_timeout != 0.0) {
    st = autotune(p, tuning_timeout, &params);
    have = (st == ST_OK);
  } else {
    have = autotune_cache_lookup(p, &params);
  }
  if (!have) params = TileParams();
  st = plan_tiles(p, params);
  if (st != ST_OK && have) st = plan_tiles(p, TileParams());
  if (st != ST_OK) {
    plan_free_tables(p);
    delete p;
    return st;
  }
  *plan = reinterpret_cast<hptt_cuda_plan_t>(p);
  return HPTT_OK;
}

int hptt_cuda_plan_exec(hptt_cuda_plan_t plan) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  return plan_enqueue(p, p->stream);
}

int hptt_cuda_plan_exec_on(hptt_cuda_plan_t plan, void *stream) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  return plan_enqueue(p, static_cast<cudaStream_t>(stream));
}

int hptt_cuda_plan_reset_data(hptt_cuda_plan_t plan, const void *in, void *out) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  p->args.A = in;
  p->args.B = out;
  return HPTT_OK;
}

int hptt_cuda_plan_describe(hptt_cuda_plan_t plan, char *buf, size_t len) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  std::string s = describe(p->args.p, p->args.t);
  char line[160];
  std::snprintf(line, sizeof(line), "grid: %d CTAs on %d SMs%s\n", p->grid, p->sm_count,
                p->tuned ? " (autotuned)" : "");
  s += line;
  if (buf && len) {
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = '\0';
  }
  return HPTT_OK;
}

int hptt_cuda_plan_set_thread_ids(hptt_cuda_plan_t plan, const int32_t *, uint32_t) {
  return plan_valid(reinterpret_cast<Plan *>(plan)) ? HPTT_OK : HPTT_ERR_HANDLE;
}

int hptt_cuda_plan_unset_thread_ids(hptt_cuda_plan_t plan) {
  return plan_valid(reinterpret_cast<Plan *>(plan)) ? HPTT_OK : HPTT_ERR_HANDLE;
}

int hptt_cuda_plan_set_stream(hptt_cuda_plan_t plan, void *stream) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  p->stream = static_cast<cudaStream_t>(stream);
  return HPTT_OK;
}

int hptt_cuda_plan_sync(hptt_cuda_plan_t plan) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  return cudaStreamSynchronize(p->stream) == cudaSuccess ? HPTT_OK : HPTT_ERR_CUDA;
}

int hptt_cuda_plan_set_coef(hptt_cuda_plan_t plan, const double *alpha,
                            const double *beta, int complex_scalars) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  if (!alpha || !beta) return HPTT_ERR_SIZE_VALUE;
  const int old_update = p->args.update;
  set_scalars(&p->args, alpha, beta, complex_scalars);
  if (p->args.update == old_update) return HPTT_OK;
  // Whether B is read changes the tile shape (per-thread iterations): plan
  // the tiles again on the plan's device.
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return HPTT_ERR_NO_DEVICE;
  if (cur != p->device && cudaSetDevice(p->device) != cudaSuccess) return HPTT_ERR_CUDA;
  TileParams params;
  if (!autotune_cache_lookup(p, &params)) params = TileParams();
  int st = plan_tiles(p, params);
  if (st != ST_OK) st = plan_tiles(p, TileParams());
  if (cur != p->device) cudaSetDevice(cur);
  return st;
}

int hptt_cuda_plan_bytes(hptt_cuda_plan_t plan, uint64_t *bytes) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p) || !bytes) return HPTT_ERR_HANDLE;
  const uint64_t sz = static_cast<uint64_t>(elem_bytes(p->args.p.dtype));
  *bytes = p->elements * sz * (p->args.update ? 3u : 2u);
  return HPTT_OK;
}

int hptt_cuda_plan_launches(hptt_cuda_plan_t plan, uint32_t *launches) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p) || !launches) return HPTT_ERR_HANDLE;
  *launches = p->args.t.num_tiles ? 1u : 0u;
  return HPTT_OK;
}

int hptt_cuda_plan_destroy(hptt_cuda_plan_t plan) {
  Plan *p = reinterpret_cast<Plan *>(plan);
  if (!plan_valid(p)) return HPTT_ERR_HANDLE;
  p->magic = 0;
  plan_free_tables(p);
  delete p;
  return HPTT_OK;
}

int hptt_cuda_plan_inspect(int dtype, uint32_t rank, const uint32_t *in_size,
                           const uint32_t *perm, const uint32_t *in_outer,
                           const uint32_t *out_outer, char *buf, size_t len) {
  if (elem_bytes(dtype) == 0) return HPTT_ERR_DTYPE;
  int st = validate(static_cast<int>(rank), in_size, perm, in_outer, out_outer,
                    in_outer ? static_cast<int>(rank) : 0,
                    out_outer ? static_cast<int>(rank) : 0);
  if (st != ST_OK) return st;
  HpttProblem p;
  st = fuse(dtype, static_cast<int>(rank), in_size, perm, in_outer, out_outer, &p);
  if (st != ST_OK) return st;
  HpttTile t;
  st = choose_tile(p, TileParams(), 0, &t);
  if (st != ST_OK) return st;
  const std::string s = describe(p, t);
  if (buf && len) {
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = '\0';
  }
  return HPTT_OK;
}

int hptt_cuda_tune_cache_load(const char *path) { return autotune_cache_load(path); }

int hptt_cuda_tune_cache_save(const char *path) { return autotune_cache_save(path); }

int hptt_cuda_tune_cache_clear(void) {
  autotune_cache_clear();
  return HPTT_OK;
}

int hptt_cuda_tune_cache_size(uint32_t *count) {
  if (!count) return HPTT_ERR_HANDLE;
  *count = static_cast<uint32_t>(autotune_cache_size());
  return HPTT_OK;
}

const char *hptt_cuda_status_string(int status) { return status_string(status); }

const char *hptt_cuda_version(void) { return "hptt-b200 0.1 (sm_100a)"; }

}  // extern "C"
