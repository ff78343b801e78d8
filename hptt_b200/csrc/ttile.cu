// TMA tile kernels (KIND_TTILE, ttile.cuh), their tensor maps and launcher.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "../../include/hptt_cuda.h"
#include "launch.h"
#include "planner.h"
#include "ttile.cuh"

namespace hptt_b200 {

using namespace dev;

namespace {

// CTAs whose bounded wait (ttile_wait) ran out, counted on each device since
// the library was loaded, read by hptt_cuda_debug_tma_timeouts.  A timed-out
// CTA stores nothing.
__device__ unsigned int g_ttile_timeouts = 0;

// try_wait polls before a CTA gives up on its loads.
constexpr uint32_t kWaitPolls = 1u << 22;

// Threads of the persistent form: at most 4 boxes of 64 consumer threads,
// and the producer warp.
constexpr int kTtilePipeThreads = 4 * 64 + 32;

// Transposes box g of a tile in shared memory: A's box (rows along the
// output's leading dim) at `ba`, the output box (rows along input dim 0) at
// `bo`, B's old box at `bb` when B is read (UPD).  64 threads per box.
template <typename E, int MODE, bool UPD>
__device__ __forceinline__ void ttile_box(const Op<E, MODE, UPD> &op, int t,
                                          const unsigned char *ba, const unsigned char *bb,
                                          unsigned char *bo) {
  constexpr int M = 16 / sizeof(E);
  const uint32_t xb = t & 7, yb = ((t & 7) + (t >> 3)) & 7;
  Vec<E, M> rows[M];
#pragma unroll
  for (int i = 0; i < M; ++i)
    rows[i] = *reinterpret_cast<const Vec<E, M> *>(ba + ttile_swz(M * yb + i, xb));
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const uint32_t o = ttile_swz(M * xb + j, yb);
    Vec<E, M> old;
    if (UPD) old = *reinterpret_cast<const Vec<E, M> *>(bb + o);
    Vec<E, M> out;
#pragma unroll
    for (int i = 0; i < M; ++i) out.v[i] = op(rows[i].v[j], UPD ? old.v[i] : rows[i].v[j]);
    *reinterpret_cast<Vec<E, M> *>(bo + o) = out;
  }
}

template <typename E, int MODE, bool UPD>
__global__ void __launch_bounds__(512)
    k_ttile(const __grid_constant__ HpttArgs args, const __grid_constant__ CUtensorMap mapA,
            const __grid_constant__ CUtensorMap mapB) {
  // programmatic dependent launch: as in k_tile (kernels.cu)
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  constexpr int BOX = 128 / sizeof(E);        // box side in elements
  constexpr uint32_t BOXB = 128u * BOX;       // box bytes
  // dynamic shared memory only (a static variable would lower the dynamic
  // limit the launcher sets to the device's opt-in maximum): the mbarrier at
  // the base, then A's and B's boxes from the next 1024-byte boundary
  // (smem_bytes = 2 K BOXB + 1024 + 16)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const HpttTile &T = args.t;
  const int K = T.tkx * T.tky;
  unsigned char *bufA = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 16 + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char *bufB = bufA + K * BOXB;
  const uint32_t sbar = smem_addr(smem_raw);
  const int tid = threadIdx.x;
  const int rank = args.p.rank;
  const int p0 = args.p.perm[0];
  int32_t org[5];
  ttile_coords(T, blockIdx.x, org);
  // box g of the tile: its A coordinates (input order) and B coordinates
  // (output order); boxes that start past the tensor's edge are skipped
  auto box = [&](int g, int32_t *ca, int32_t *cb) -> bool {
    for (int d = 0; d < 5; ++d) ca[d] = org[d];
    ca[0] += (g % T.tkx) * BOX;
    ca[p0] += (g / T.tkx) * BOX;
    for (int k = 0; k < 5; ++k) cb[k] = k < rank ? ca[args.p.perm[k]] : 0;
    return ca[0] < args.p.n[0] && ca[p0] < args.p.n[p0];
  };
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    int nvalid = 0;
    for (int g = 0; g < K; ++g) {
      int32_t ca[5], cb[5];
      nvalid += box(g, ca, cb) ? 1 : 0;
    }
    const uint32_t bytes = nvalid * BOXB * (UPD ? 2u : 1u);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sbar),
                 "r"(bytes)
                 : "memory");
    for (int g = 0; g < K; ++g) {
      int32_t ca[5], cb[5];
      if (!box(g, ca, cb)) continue;
      ttile_load(&mapA, smem_addr(bufA + g * BOXB), sbar, rank, ca);
      if (UPD) ttile_load(&mapB, smem_addr(bufB + g * BOXB), sbar, rank, cb);
    }
  }
  // every thread waits; if any gave up, the whole CTA stores nothing, and
  // thread 0 waits once more (bounded) for the loads still in flight
  const bool timed_out = !ttile_wait(sbar, 0, kWaitPolls);
  if (__syncthreads_or(timed_out)) {
    if (tid == 0) {
      atomicAdd(&g_ttile_timeouts, 1u);
      ttile_wait(sbar, 0, kWaitPolls);
    }
    return;
  }
  const Scal sc{args.alpha[0], args.alpha[1], args.beta[0], args.beta[1]};
  const Op<E, MODE, UPD> op(sc);
  const int g = tid >> 6;
  // in place: each thread reads B's old values and writes the results at
  // the same 16-byte rows of the B-side box
  if (g < K)
    ttile_box<E, MODE, UPD>(op, tid & 63, bufA + g * BOXB, bufB + g * BOXB, bufB + g * BOXB);
  // the generic-proxy writes above must be visible to the TMA stores
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  if (tid == 0) {
    for (int gg = 0; gg < K; ++gg) {
      int32_t ca[5], cb[5];
      if (!box(gg, ca, cb)) continue;
      ttile_store(&mapB, smem_addr(bufB + gg * BOXB), rank, cb);
    }
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
  }
}

// Persistent form (ttile.cuh): CTAs walk tiles blockIdx.x + i * gridDim.x.
// Warp-specialised: the last warp's lane 0 produces (arms stage i % S and
// loads tile i once the consumers have released the stage), the first 64 K
// threads consume (transpose, then their thread 0 issues the stores and
// releases the stage).  Shared memory: 2 S mbarriers (full, empty) and S
// tile origins in a 256-byte header, then from the next 1024-byte boundary
// the S stages (K A boxes, then K B boxes when B is read) and three output
// buffers (smem_bytes = S * stage + 3 K BOXB + 1024 + 256).
template <typename E, int MODE, bool UPD>
__global__ void __launch_bounds__(kTtilePipeThreads)
    k_ttile_pipe(const __grid_constant__ HpttArgs args, const __grid_constant__ CUtensorMap mapA,
                 const __grid_constant__ CUtensorMap mapB) {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  constexpr int BOX = 128 / sizeof(E);
  constexpr uint32_t BOXB = 128u * BOX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const HpttTile &T = args.t;
  const int K = T.tkx * T.tky;
  const int S = T.ts;
  const int nc = 64 * K;  // consumer threads
  const uint32_t stage_bytes = K * BOXB * (UPD ? 2u : 1u);
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 256 + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char *obuf = base + S * stage_bytes;
  const uint32_t full0 = smem_addr(smem_raw);    // full[s] at full0 + 8 s
  const uint32_t empty0 = full0 + 64;            // empty[s] at empty0 + 8 s
  int32_t *origin = reinterpret_cast<int32_t *>(smem_raw + 128);  // [S][5]
  const int tid = threadIdx.x;
  const int rank = args.p.rank;
  const int p0 = args.p.perm[0];
  const uint32_t step = gridDim.x;
  const uint32_t mine =
      blockIdx.x < T.num_tiles ? (T.num_tiles - blockIdx.x + step - 1) / step : 0;
  // box g of a tile with origin `org`: A coordinates (input order), B
  // coordinates (output order); false for a box that starts past the edge
  auto box = [&](const int32_t *org, int g, int32_t *ca, int32_t *cb) -> bool {
    for (int d = 0; d < 5; ++d) ca[d] = org[d];
    ca[0] += (g % T.tkx) * BOX;
    ca[p0] += (g / T.tkx) * BOX;
    for (int k = 0; k < 5; ++k) cb[k] = k < rank ? ca[args.p.perm[k]] : 0;
    return ca[0] < args.p.n[0] && ca[p0] < args.p.n[p0];
  };
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full0 + 8u * s) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty0 + 8u * s) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid >= nc) {
    // producer
    if (tid != nc) return;
    for (uint32_t i = 0; i < mine; ++i) {
      const int s = static_cast<int>(i % S);
      if (i >= static_cast<uint32_t>(S) &&
          !ttile_wait(empty0 + 8u * s, (i / S - 1) & 1u, kWaitPolls)) {
        atomicAdd(&g_ttile_timeouts, 1u);
        return;  // the consumers' waits for this stage run out in turn
      }
      int32_t *org = origin + 5 * s;
      ttile_coords(T, blockIdx.x + i * step, org);
      int nvalid = 0;
      for (int g = 0; g < K; ++g) {
        int32_t ca[5], cb[5];
        nvalid += box(org, g, ca, cb) ? 1 : 0;
      }
      const uint32_t bar = full0 + 8u * s;
      // the arrive releases the origin written above to the consumers
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                   "r"(nvalid * BOXB * (UPD ? 2u : 1u))
                   : "memory");
      unsigned char *st = base + s * stage_bytes;
      for (int g = 0; g < K; ++g) {
        int32_t ca[5], cb[5];
        if (!box(org, g, ca, cb)) continue;
        ttile_load(&mapA, smem_addr(st + g * BOXB), bar, rank, ca);
        if (UPD) ttile_load(&mapB, smem_addr(st + (K + g) * BOXB), bar, rank, cb);
      }
    }
    return;
  }
  // consumers
  const Scal sc{args.alpha[0], args.alpha[1], args.beta[0], args.beta[1]};
  const Op<E, MODE, UPD> op(sc);
  const int g = tid >> 6;
  uint32_t i = 0;
  bool timed_out = false;
  for (; i < mine; ++i) {
    const int s = static_cast<int>(i % S);
    const bool ok = ttile_wait(full0 + 8u * s, (i / S) & 1u, kWaitPolls);
    unsigned char *st = base + s * stage_bytes;
    unsigned char *ob = obuf + (i % 3u) * K * BOXB;
    // output buffer i % 3 was last read by the stores of tile i - 3, done
    // (wait_group.read 1 before the barrier of tile i - 1)
    if (ok)
      ttile_box<E, MODE, UPD>(op, tid & 63, st + g * BOXB, st + (K + g) * BOXB, ob + g * BOXB);
    // the generic-proxy writes above must be visible to the TMA stores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    // stores of tile i - 2 have read their buffer before the consumers pass
    // this barrier (so tile i + 1 may write it)
    if (tid == 0) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
    uint32_t any_bad = 0;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n"
        " barrier.red.or.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(any_bad)
        : "r"(ok ? 0u : 1u), "r"(nc)
        : "memory");
    if (any_bad) {
      timed_out = true;
      break;
    }
    if (tid == 0) {
      const int32_t *org = origin + 5 * s;
      for (int gg = 0; gg < K; ++gg) {
        int32_t ca[5], cb[5];
        if (!box(org, gg, ca, cb)) continue;
        ttile_store(&mapB, smem_addr(ob + gg * BOXB), rank, cb);
      }
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
      // stage s is free: every consumer passed the barrier after reading it
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(empty0 + 8u * s)
                   : "memory");
    }
  }
  if (tid == 0) {
    if (timed_out) {
      atomicAdd(&g_ttile_timeouts, 1u);
      // loads the producer may still have in flight (tiles i .. i + S - 1),
      // each wait bounded
      for (uint32_t j = i + 1; j < i + S && j < mine; ++j)
        ttile_wait(full0 + 8u * (j % S), (j / S) & 1u, kWaitPolls);
    }
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
  }
}

template <typename E, int MODE, bool UPD>
const void *kptr(bool pipe) {
  return pipe ? reinterpret_cast<const void *>(&k_ttile_pipe<E, MODE, UPD>)
              : reinterpret_cast<const void *>(&k_ttile<E, MODE, UPD>);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// Tensor map of one side (0: A in input order, 1: B in output order).
cudaError_t encode(const HpttProblem &P, const HpttTile &T, int side, const void *base,
                   CUtensorMap *map) {
  TtileMapParams mp;
  if (ttile_map_params(P, T, side, &mp) != ST_OK) return cudaErrorInvalidValue;
  const auto fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  cuuint64_t dims[5], strides[4];
  cuuint32_t boxd[5], elem[5];
  for (int k = 0; k < mp.rank; ++k) {
    dims[k] = mp.dims[k];
    boxd[k] = mp.box[k];
    elem[k] = 1;
    if (k > 0) strides[k - 1] = mp.stride_bytes[k];
  }
  const CUtensorMapDataType dt =
      mp.elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_UINT64;
  const CUresult r = fn(map, dt, static_cast<cuuint32_t>(mp.rank), const_cast<void *>(base), dims,
                        strides, boxd, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace

const void *ttile_kernel_for(const HpttArgs &a) {
  const bool upd = a.update != 0;
  const bool copy = a.mode == MODE_COPY && !upd;
  const bool pp = a.t.ts != 0;
  switch (a.p.dtype) {
    case DT_F32:
      if (copy) return kptr<unsigned int, MODE_COPY, false>(pp);
      if (a.mode == MODE_CPLX) return nullptr;
      return upd ? kptr<float, MODE_REAL, true>(pp) : kptr<float, MODE_REAL, false>(pp);
    case DT_F64:
      if (copy) return kptr<unsigned long long, MODE_COPY, false>(pp);
      if (a.mode == MODE_CPLX) return nullptr;
      return upd ? kptr<double, MODE_REAL, true>(pp) : kptr<double, MODE_REAL, false>(pp);
    case DT_C64:
      if (copy) return kptr<unsigned long long, MODE_COPY, false>(pp);
      if (a.mode == MODE_CPLX)
        return upd ? kptr<float2, MODE_CPLX, true>(pp) : kptr<float2, MODE_CPLX, false>(pp);
      return upd ? kptr<float2, MODE_REAL, true>(pp) : kptr<float2, MODE_REAL, false>(pp);
    default:
      return nullptr;
  }
}

cudaError_t launch_ttile(const HpttArgs &a, int grid, cudaStream_t stream) {
  const void *fn = ttile_kernel_for(a);
  if (!fn) return cudaErrorInvalidValue;
  if (a.t.num_tiles == 0) return cudaSuccess;
  // TMA needs 16-byte aligned bases (the planner checked the strides)
  if ((reinterpret_cast<uintptr_t>(a.A) | reinterpret_cast<uintptr_t>(a.B)) & 15)
    return cudaErrorMisalignedAddress;
  alignas(64) CUtensorMap mapA, mapB;
  cudaError_t e = encode(a.p, a.t, 0, a.A, &mapA);
  if (e == cudaSuccess) e = encode(a.p, a.t, 1, a.B, &mapB);
  if (e != cudaSuccess) return e;
  void *params[] = {const_cast<HpttArgs *>(&a), &mapA, &mapB};
  cudaLaunchConfig_t cfg = {};
  // one CTA per tile, or the persistent grid (resident CTAs, at most one
  // per tile)
  uint32_t ctas = a.t.num_tiles;
  if (a.t.ts && grid > 0 && static_cast<uint32_t>(grid) < ctas) ctas = static_cast<uint32_t>(grid);
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(a.t.nt);
  cfg.dynamicSmemBytes = static_cast<size_t>(a.t.smem_bytes);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, params);
}

}  // namespace hptt_b200

using namespace hptt_b200;

extern "C" int hptt_cuda_debug_tma_timeouts(uint32_t *count) {
  if (!count) return HPTT_ERR_HANDLE;
  unsigned int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_ttile_timeouts, sizeof(v)) != cudaSuccess) {
    cudaGetLastError();
    return HPTT_ERR_CUDA;
  }
  *count = v;
  return HPTT_OK;
}
