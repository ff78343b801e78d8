// Allocation-free transpose entry point.
//
// hptt_cuda_plan_create keeps each plan's offset tables (a few KB) in a
// device buffer it obtains with cudaMalloc.  Some callers cannot allocate
// device memory at the moment they need a transpose: runtimes whose device
// memory is handed out only by their own pool or arena (a cudaMalloc behind
// the pool's back would break its accounting or fail under its reservation),
// and jobs held to a fixed device-memory budget.  hptt_cuda_transpose_noalloc
// serves them: it plans on the host, copies the tables into a fixed array
// compiled into this library, and launches the same kernel -- without
// cudaMalloc, cudaFree or any other device allocator.
//
// The array is a file-scope __device__ variable of HPTT_NOALLOC_TABLE_BYTES
// bytes; every GPU that loads the library holds it until the process exits.
// In host code its name only stands in for it, so every call looks its
// device address up in the current context with cudaGetSymbolAddress, and
// that address is what the kernel receives (so the call keeps working after
// cudaDeviceReset re-creates the context).
#include <cuda_runtime.h>

#include <vector>

#include "../../include/hptt_cuda.h"
#include "autotune.h"
#include "launch.h"
#include "plan.h"
#include "planner.h"
#include "tables.h"

namespace hptt_b200 {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_tables[HPTT_NOALLOC_TABLE_BYTES];

// Device address of g_noalloc_tables in the current context, looked up on
// every call (a host-side query; a cached address would outlive a context
// torn down by cudaDeviceReset).
int table_address(int device, void **out) {
  if (device < 0) return ST_NO_DEVICE;
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_tables);
  if (e != cudaSuccess || !ptr) {
    cudaGetLastError();
    return ST_CUDA;
  }
  *out = ptr;
  return ST_OK;
}

}  // namespace
}  // namespace hptt_b200

using namespace hptt_b200;

extern "C" int hptt_cuda_transpose_noalloc(int dtype, uint32_t rank, const uint32_t *in_size,
                                           const uint32_t *perm, const uint32_t *in_outer,
                                           const uint32_t *out_outer, const double *alpha,
                                           const double *beta, int complex_scalars,
                                           const void *in, void *out, void *stream) {
  // the same argument guard as hptt_cuda_plan_create
  if (!in || !out) return HPTT_ERR_NULL_DATA;
  if (elem_bytes(dtype) == 0) return HPTT_ERR_DTYPE;
  int st = validate(static_cast<int>(rank), in_size, perm, in_outer, out_outer,
                    in_outer ? static_cast<int>(rank) : 0,
                    out_outer ? static_cast<int>(rank) : 0);
  if (st != ST_OK) return st;
  if (!alpha || !beta) return HPTT_ERR_SIZE_VALUE;

  HpttArgs a{};
  st = fuse(dtype, static_cast<int>(rank), in_size, perm, in_outer, out_outer, &a.p);
  if (st != ST_OK) return st;
  a.A = in;
  a.B = out;
  set_scalars(&a, alpha, beta, complex_scalars);

  // The tile the plan path would run: the autotune cache's entry for this
  // problem when there is one (its key needs only the fused problem, the
  // element count and whether B is read), else the planner's default.  An
  // entry whose tables would not fit the array falls back to the default.
  TileParams tp;
  {
    Plan probe;
    probe.args = a;
    probe.elements = 1;
    for (uint32_t d = 0; d < rank; ++d) probe.elements *= in_size[d];
    TileParams cached;
    if (autotune_cache_lookup(&probe, &cached) &&
        choose_tile(a.p, cached, a.update, &a.t) == ST_OK &&
        a.t.table_bytes <= HPTT_NOALLOC_TABLE_BYTES)
      tp = cached;
  }
  st = choose_tile(a.p, tp, a.update, &a.t);
  if (st != ST_OK) return st;
  int vec = a.t.kind == KIND_ROWS ? a.t.vec : 1;
  if (vec > 1) {
    const uintptr_t bytes = static_cast<uintptr_t>(vec) * elem_bytes(dtype);
    if (reinterpret_cast<uintptr_t>(in) % bytes || reinterpret_cast<uintptr_t>(out) % bytes) {
      tp.max_vec_bytes = elem_bytes(dtype);
      st = choose_tile(a.p, tp, a.update, &a.t);
      if (st != ST_OK) return st;
      vec = 1;
    }
  }
  if (a.t.kind == KIND_TTILE &&
      ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)) {
    // no tensor map for these bases: the element tile
    tp.tt = 0;
    tp.vt = 0;
    st = choose_tile(a.p, tp, a.update, &a.t);
    if (st != ST_OK) return st;
  }
  if (a.t.num_tiles == 0) return HPTT_OK;
  if (a.t.table_bytes > HPTT_NOALLOC_TABLE_BYTES) return HPTT_ERR_TOO_LARGE;

  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return HPTT_ERR_NO_DEVICE;
  void *tables = nullptr;
  st = table_address(device, &tables);
  if (st != ST_OK) return st;

  // Every byte the kernel reads is rewritten below, so nothing in the array
  // has to start at zero.  The source is pageable host memory: the copy
  // returns once the bytes are staged and is ordered before the launch.
  std::vector<unsigned char> host;
  build_tables(a.p, a.t, &host);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(tables, host.data(), host.size(), cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return HPTT_ERR_CUDA;
  a.tables = tables;
  int per_sm = 0, sms = 0;
  if (occupancy(a, vec, &per_sm) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return HPTT_ERR_CUDA;
  // the persistent TMA tile's grid: the resident CTAs (other kernels run one
  // CTA per tile)
  if (launch_single(a, vec, per_sm * sms, s) != cudaSuccess) return HPTT_ERR_CUDA;
  return HPTT_OK;
}

extern "C" size_t hptt_cuda_noalloc_table_bytes(void) { return HPTT_NOALLOC_TABLE_BYTES; }
