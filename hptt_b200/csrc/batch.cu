// Batched form: the group kernels and their host side (see batch.h).
#include "batch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <utility>

#include "../../include/hptt_cuda.h"
#include "kernels.cuh"
#include "plan.h"
#include "planner.h"

namespace hptt_b200 {

using namespace dev;

namespace {

constexpr int kNT = kBatchThreads;
// Tile bodies ("shapes"):
//   0 tile, table offsets (uint32)      3 rows, widest vector (uint32)
//   1 tile, single-dim sides (uint32)   4 rows, scalar (uint32)
//   2 tile, table offsets (int64)       5 rows, scalar (int64)
constexpr int kShapes = 6;
// Element storage and arithmetic ("combos"), the same choices as the
// single-transpose kernels (kernels.cu: kernel_for):
//   0 f32 copy   1 8-byte copy   2 16-byte copy
//   3/4 f32 scale / update        5/6 f64 scale / update
//   7/8 c64 real scalars          9/10 c64 complex scalars
//   11/12 c128 real scalars       13/14 c128 complex scalars
constexpr int kCombos = 15;
constexpr int kBodies = kCombos * kShapes;

template <typename E>
constexpr int vmax_rows() {
  return sizeof(E) == 4 ? 4 : (sizeof(E) == 8 ? 2 : 1);
}

// Resident-CTA targets: 4 (64 registers) for every tile body -- the
// persistent loop keeps its own state live across the body, so 4 of the 40
// tile bodies spill 44-64 bytes; on the 4096-transpose mixed batch this ran
// 5 % faster than 3 CTAs (80 registers, no spills), and 5 CTAs spilled up to
// 220 bytes in most bodies; rows bodies are not bounded.
template <bool UPD, int SHAPE>
constexpr int min_ctas() {
  return SHAPE >= 3 ? 1 : 4;
}

// Persistent kernel of one group: CTAs take items [begin, end) of the work
// list from *counter.  The item's descriptor is staged in shared memory (one
// coalesced copy); consecutive tiles reuse the tile buffer, hence the
// barriers.
template <typename E, int MODE, bool UPD, int SHAPE>
__global__ void __launch_bounds__(kNT, (min_ctas<UPD, SHAPE>()))
    k_batch(const HpttBatchDesc *__restrict__ descs, const HpttWork *__restrict__ work,
            uint32_t begin, uint32_t end, uint32_t *__restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(16) HpttBatchDesc sd;
  __shared__ uint32_t s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = begin + atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t it = s_item;
    if (it >= end) break;
    const HpttWork w = work[it];
    {
      const int4 *src = reinterpret_cast<const int4 *>(descs + w.desc);
      int4 *dst = reinterpret_cast<int4 *>(&sd);
      for (int i = threadIdx.x; i < static_cast<int>(sizeof(HpttBatchDesc) / 16); i += kNT)
        dst[i] = src[i];
    }
    __syncthreads();
    const HpttArgs &a = sd.a;
    const Scal sc{a.alpha[0], a.alpha[1], a.beta[0], a.beta[1]};
    const Op<E, MODE, UPD> op(sc);
    const E *A = static_cast<const E *>(a.A);
    E *B = static_cast<E *>(a.B);
    const unsigned char *tab = static_cast<const unsigned char *>(a.tables);
    for (uint32_t k = 0; k < w.ntiles; ++k) {
      const uint32_t tile = w.tile0 + k;
      if (SHAPE <= 2) {
        if (k) __syncthreads();
        E *s = reinterpret_cast<E *>(smem);
        if (SHAPE == 0)
          tile_one<E, MODE, UPD, uint32_t, false, false, false>(a.p, a.t, A, B, tab, op, s, tile);
        else if (SHAPE == 1)
          tile_one<E, MODE, UPD, uint32_t, true, true, false>(a.p, a.t, A, B, tab, op, s, tile);
        else
          tile_one<E, MODE, UPD, int64_t, false, false, false>(a.p, a.t, A, B, tab, op, s, tile);
      } else if (SHAPE == 3) {
        rows_one<E, MODE, UPD, uint32_t, vmax_rows<E>()>(a.p, a.t, A, B, tab, op, tile);
      } else if (SHAPE == 4) {
        rows_one<E, MODE, UPD, uint32_t, 1>(a.p, a.t, A, B, tab, op, tile);
      } else {
        rows_one<E, MODE, UPD, int64_t, 1>(a.p, a.t, A, B, tab, op, tile);
      }
    }
    __syncthreads();
  }
}

template <typename E, int MODE, bool UPD>
const void *kernel_shape(int shape) {
  switch (shape) {
    case 0: return reinterpret_cast<const void *>(&k_batch<E, MODE, UPD, 0>);
    case 1: return reinterpret_cast<const void *>(&k_batch<E, MODE, UPD, 1>);
    case 2: return reinterpret_cast<const void *>(&k_batch<E, MODE, UPD, 2>);
    case 3: return reinterpret_cast<const void *>(&k_batch<E, MODE, UPD, 3>);
    case 4: return reinterpret_cast<const void *>(&k_batch<E, MODE, UPD, 4>);
    default: return reinterpret_cast<const void *>(&k_batch<E, MODE, UPD, 5>);
  }
}

const void *kernel_of(int body) {
  const int shape = body % kShapes;
  switch (body / kShapes) {
    case 0: return kernel_shape<unsigned int, MODE_COPY, false>(shape);
    case 1: return kernel_shape<unsigned long long, MODE_COPY, false>(shape);
    case 2: return kernel_shape<uint4, MODE_COPY, false>(shape);
    case 3: return kernel_shape<float, MODE_REAL, false>(shape);
    case 4: return kernel_shape<float, MODE_REAL, true>(shape);
    case 5: return kernel_shape<double, MODE_REAL, false>(shape);
    case 6: return kernel_shape<double, MODE_REAL, true>(shape);
    case 7: return kernel_shape<float2, MODE_REAL, false>(shape);
    case 8: return kernel_shape<float2, MODE_REAL, true>(shape);
    case 9: return kernel_shape<float2, MODE_CPLX, false>(shape);
    case 10: return kernel_shape<float2, MODE_CPLX, true>(shape);
    case 11: return kernel_shape<double2, MODE_REAL, false>(shape);
    case 12: return kernel_shape<double2, MODE_REAL, true>(shape);
    case 13: return kernel_shape<double2, MODE_CPLX, false>(shape);
    case 14: return kernel_shape<double2, MODE_CPLX, true>(shape);
    default: return nullptr;
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
int combo_of(const HpttArgs &a) {
  const bool upd = a.update != 0;
  const bool copy = a.mode == MODE_COPY && !upd;
  switch (a.p.dtype) {
    case DT_F32: return copy ? 0 : (upd ? 4 : 3);
    case DT_F64: return copy ? 1 : (upd ? 6 : 5);
    case DT_C64:
      if (copy) return 1;
      if (a.mode == MODE_CPLX) return upd ? 10 : 9;
      return upd ? 8 : 7;
    case DT_C128:
      if (copy) return 2;
      if (a.mode == MODE_CPLX) return upd ? 14 : 13;
      return upd ? 12 : 11;
    default: return -1;
  }
}

int vmax_for(int dtype) {
  const int s = elem_bytes(dtype);
  return s == 4 ? 4 : (s == 8 ? 2 : 1);
}

// Shape body for a tile and vector width, or -1 when none fits.
int shape_of(const HpttTile &t, int vec, int dtype) {
  if (t.kind == KIND_TILE) {
    if (t.big_offsets) return 2;
    return (t.nx <= 1 && t.ny <= 1) ? 1 : 0;
  }
  if (vec == 1) return t.big_offsets ? 5 : 4;
  if (!t.big_offsets && vec == vmax_for(dtype)) return 3;
  return -1;
}

// Resident CTAs per SM of a group kernel with `smem` dynamic bytes (cached:
// the attribute call and the occupancy query cost microseconds, and the
// served form asks for every launch).
int group_occupancy(int body, int smem, int *per_sm) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ST_CUDA;
  const auto key = std::make_pair(body * 64 + dev, smem);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      *per_sm = it->second;
      return ST_OK;
    }
  }
  const void *fn = kernel_of(body);
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return ST_CUDA;
  const int static_smem = static_cast<int>(sizeof(HpttBatchDesc)) + 16;
  if (smem + static_smem > optin) return ST_TOO_LARGE;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           optin - static_smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, kNT,
                                                    static_cast<size_t>(smem)) != cudaSuccess)
    return ST_CUDA;
  std::lock_guard<std::mutex> lk(mu);
  cache[key] = *per_sm;
  return ST_OK;
}

}  // namespace

bool batch_valid(const Batch *b) { return b && b->magic == kBatchMagic; }

int batch_layout(const std::vector<BatchEntry> &entries, int sms, BatchLayout *L) {
  const size_t n = entries.size();
  L->desc.assign(n, HpttBatchDesc{});
  L->work.clear();
  L->groups.clear();
  L->bytes = 0;
  std::vector<std::vector<uint32_t>> by_body(kBodies);
  for (size_t i = 0; i < n; ++i) {
    const Plan *p = entries[i].plan;
    if (!plan_valid(p)) return ST_BAD_HANDLE;
    HpttBatchDesc &d = L->desc[i];
    d.a = p->args;
    if (entries[i].A || entries[i].B) {
      d.a.A = entries[i].A;
      d.a.B = entries[i].B;
    }
    if (!d.a.A || !d.a.B) return ST_NULL_DATA;
    // the plan's vector tile when the pointers allow it (plan_vec_for_ptrs)
    int vec = p->vec;
    if (vec > 1) {
      const uintptr_t vb = static_cast<uintptr_t>(vec) * elem_bytes(d.a.p.dtype);
      if (reinterpret_cast<uintptr_t>(d.a.A) % vb || reinterpret_cast<uintptr_t>(d.a.B) % vb)
        vec = 1;
    }
    if (vec == p->vec) {
      d.a.tables = p->dtab;
    } else {
      d.a.t = p->tile_scalar;
      d.a.tables = p->dtab_scalar;
    }
    if (d.a.t.nt != kNT || d.a.t.kind == KIND_VTILE || d.a.t.kind == KIND_TTILE) {
      // a 512-thread, vector-tile or TMA-tile plan: its tile planned for the
      // batch kernels' 256-thread tile form
      d.a.t = p->tile_batch;
      d.a.tables = p->dtab_batch;
      vec = 1;
    }
    int shape = shape_of(d.a.t, vec, d.a.p.dtype);
    if (shape < 0) {
      // a rows vector width without a batch body: the plan's scalar tile
      d.a.t = p->tile_scalar;
      d.a.tables = p->dtab_scalar;
      vec = 1;
      shape = shape_of(d.a.t, vec, d.a.p.dtype);
    }
    const int combo = combo_of(d.a);
    if (combo < 0 || shape < 0) return ST_BAD_DTYPE;
    d.body = combo * kShapes + shape;
    d.vec = vec;
    L->bytes += p->elements * static_cast<uint64_t>(elem_bytes(d.a.p.dtype)) *
                (d.a.update ? 3u : 2u);
    if (d.a.t.num_tiles) by_body[d.body].push_back(static_cast<uint32_t>(i));
  }
  // groups, their grids and the work list (items of up to kBatchChunkMax
  // tiles, small enough that every CTA of the group takes several)
  for (int body = 0; body < kBodies; ++body) {
    if (by_body[body].empty()) continue;
    BatchGroup g;
    g.body = body;
    uint64_t tiles = 0;
    for (uint32_t i : by_body[body]) {
      g.smem_bytes = std::max(g.smem_bytes, L->desc[i].a.t.smem_bytes);
      tiles += L->desc[i].a.t.num_tiles;
    }
    int per_sm = 0;
    const int st = group_occupancy(body, g.smem_bytes, &per_sm);
    if (st != ST_OK) return st;
    if (per_sm < 1) return ST_TOO_LARGE;
    const uint64_t full = static_cast<uint64_t>(per_sm) * sms;
    const uint64_t chunk =
        std::max<uint64_t>(1, std::min<uint64_t>(kBatchChunkMax, tiles / (8 * full)));
    g.begin = static_cast<uint32_t>(L->work.size());
    for (uint32_t i : by_body[body]) {
      const uint32_t nt = L->desc[i].a.t.num_tiles;
      for (uint32_t t0 = 0; t0 < nt; t0 += static_cast<uint32_t>(chunk))
        L->work.push_back(HpttWork{i, t0,
                                   static_cast<uint32_t>(std::min<uint64_t>(chunk, nt - t0)), 0});
    }
    g.end = static_cast<uint32_t>(L->work.size());
    g.grid = static_cast<int>(std::min<uint64_t>(full, g.end - g.begin));
    L->groups.push_back(g);
  }
  return ST_OK;
}

int batch_launch_group(const BatchGroup &g, const HpttBatchDesc *d_desc, const HpttWork *d_work,
                       uint32_t *d_counter, cudaStream_t stream) {
  const void *fn = kernel_of(g.body);
  uint32_t begin = g.begin, end = g.end;
  void *params[] = {&d_desc, &d_work, &begin, &end, &d_counter};
  return cudaLaunchKernel(fn, dim3(g.grid), dim3(kNT), params,
                          static_cast<size_t>(g.smem_bytes), stream) == cudaSuccess
             ? ST_OK
             : ST_CUDA;
}

int batch_launch_groups(const std::vector<BatchGroup> &groups, const HpttBatchDesc *d_desc,
                        const HpttWork *d_work, uint32_t *d_counters, cudaStream_t stream) {
  if (groups.empty()) return ST_OK;
  if (cudaMemsetAsync(d_counters, 0, groups.size() * sizeof(uint32_t), stream) != cudaSuccess)
    return ST_CUDA;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const int st = batch_launch_group(groups[gi], d_desc, d_work, d_counters + gi, stream);
    if (st != ST_OK) return st;
  }
  return ST_OK;
}

int batch_build(Batch *b) {
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess)
    return ST_CUDA;
  std::vector<BatchEntry> entries(b->plans.size());
  for (size_t i = 0; i < b->plans.size(); ++i) entries[i].plan = b->plans[i];
  BatchLayout L;
  const int lst = batch_layout(entries, sms, &L);
  if (lst != ST_OK) return lst;
  const size_t n = L.desc.size();
  std::vector<BatchGroup> &groups = L.groups;
  std::vector<HpttWork> &work = L.work;
  b->desc = L.desc;
  b->bytes = L.bytes;
  // the graph stays valid while groups, grids, shared memory and buffers do
  bool same = b->graph_exec && groups.size() == b->groups.size() &&
              work.size() <= b->work_capacity && groups.size() <= b->counter_capacity;
  for (size_t k = 0; same && k < groups.size(); ++k)
    same = groups[k].body == b->groups[k].body && groups[k].begin == b->groups[k].begin &&
           groups[k].end == b->groups[k].end && groups[k].grid == b->groups[k].grid &&
           groups[k].smem_bytes == b->groups[k].smem_bytes;
  b->groups = groups;
  b->work = work;
  if (!b->d_desc && n) {
    if (cudaMalloc(&b->d_desc, n * sizeof(HpttBatchDesc)) != cudaSuccess) {
      cudaGetLastError();
      return ST_ALLOC;
    }
  }
  if (work.size() > b->work_capacity) {
    if (b->d_work) cudaFree(b->d_work);
    b->d_work = nullptr;
    b->work_capacity = 0;
    if (cudaMalloc(&b->d_work, work.size() * sizeof(HpttWork)) != cudaSuccess) {
      cudaGetLastError();
      return ST_ALLOC;
    }
    b->work_capacity = static_cast<uint32_t>(work.size());
  }
  if (groups.size() > b->counter_capacity) {
    if (b->d_counters) cudaFree(b->d_counters);
    b->d_counters = nullptr;
    b->counter_capacity = 0;
    if (cudaMalloc(&b->d_counters, groups.size() * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      return ST_ALLOC;
    }
    b->counter_capacity = static_cast<uint32_t>(groups.size());
  }
  if ((n && cudaMemcpy(b->d_desc, b->desc.data(), n * sizeof(HpttBatchDesc),
                       cudaMemcpyHostToDevice) != cudaSuccess) ||
      (!work.empty() && cudaMemcpy(b->d_work, work.data(), work.size() * sizeof(HpttWork),
                                   cudaMemcpyHostToDevice) != cudaSuccess))
    return ST_CUDA;
  if (b->graph_exec && !same) return batch_capture(b);
  return ST_OK;
}

int batch_enqueue(Batch *b, cudaStream_t stream) {
  if (b->groups.empty()) return ST_OK;
  if (b->graph_exec)
    return cudaGraphLaunch(b->graph_exec, stream) == cudaSuccess ? ST_OK : ST_CUDA;
  return batch_launch_groups(b->groups, b->d_desc, b->d_work, b->d_counters, stream);
}

int batch_capture(Batch *b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->graph_exec = nullptr;
  b->graph = nullptr;
  if (b->groups.empty()) return ST_OK;
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return ST_CUDA;
  int st = ST_OK;
  cudaGraphNode_t reset = nullptr;
  cudaMemsetParams mp = {};
  mp.dst = b->d_counters;
  mp.value = 0;
  mp.elementSize = sizeof(uint32_t);
  mp.width = b->groups.size();
  mp.height = 1;
  mp.pitch = 0;
  if (cudaGraphAddMemsetNode(&reset, g, nullptr, 0, &mp) != cudaSuccess) st = ST_CUDA;
  // the group kernels depend on the reset only, not on one another
  std::vector<void *> args(5 * b->groups.size());
  std::vector<uint32_t> ranges(2 * b->groups.size());
  std::vector<uint32_t *> counters(b->groups.size());
  const HpttBatchDesc *descs = b->d_desc;
  const HpttWork *work = b->d_work;
  for (size_t gi = 0; st == ST_OK && gi < b->groups.size(); ++gi) {
    const BatchGroup &grp = b->groups[gi];
    ranges[2 * gi] = grp.begin;
    ranges[2 * gi + 1] = grp.end;
    counters[gi] = b->d_counters + gi;
    void **a = &args[5 * gi];
    a[0] = const_cast<HpttBatchDesc **>(&descs);
    a[1] = const_cast<HpttWork **>(&work);
    a[2] = &ranges[2 * gi];
    a[3] = &ranges[2 * gi + 1];
    a[4] = &counters[gi];
    cudaKernelNodeParams kp = {};
    kp.func = const_cast<void *>(kernel_of(grp.body));
    kp.gridDim = dim3(grp.grid);
    kp.blockDim = dim3(kNT);
    kp.sharedMemBytes = static_cast<unsigned>(grp.smem_bytes);
    kp.kernelParams = a;
    cudaGraphNode_t node = nullptr;
    if (cudaGraphAddKernelNode(&node, g, &reset, 1, &kp) != cudaSuccess) st = ST_CUDA;
  }
  if (st == ST_OK && cudaGraphInstantiate(&b->graph_exec, g, 0) != cudaSuccess) {
    b->graph_exec = nullptr;
    st = ST_CUDA;
  }
  if (st == ST_OK) {
    b->graph = g;
  } else {
    cudaGraphDestroy(g);
    cudaGetLastError();
  }
  return st;
}

void batch_free(Batch *b) {
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_desc) cudaFree(b->d_desc);
  if (b->d_work) cudaFree(b->d_work);
  if (b->d_counters) cudaFree(b->d_counters);
  b->graph_exec = nullptr;
  b->graph = nullptr;
  b->d_desc = nullptr;
  b->d_work = nullptr;
  b->d_counters = nullptr;
  b->work_capacity = 0;
  b->counter_capacity = 0;
}

}  // namespace hptt_b200

using namespace hptt_b200;

extern "C" {

int hptt_cuda_batch_create(const hptt_cuda_plan_t *plans, uint32_t count,
                           hptt_cuda_batch_t *batch) {
  if (!batch) return HPTT_ERR_HANDLE;
  *batch = nullptr;
  if (count && !plans) return HPTT_ERR_HANDLE;
  for (uint32_t i = 0; i < count; ++i)
    if (!plan_valid(reinterpret_cast<Plan *>(plans[i]))) return HPTT_ERR_HANDLE;
  Batch *b = new (std::nothrow) Batch();
  if (!b) return HPTT_ERR_ALLOC;
  if (cudaGetDevice(&b->device) != cudaSuccess) {
    delete b;
    return HPTT_ERR_NO_DEVICE;
  }
  b->plans.reserve(count);
  for (uint32_t i = 0; i < count; ++i) {
    Plan *p = reinterpret_cast<Plan *>(plans[i]);
    if (p->device != b->device) {
      delete b;
      return HPTT_ERR_HANDLE;
    }
    b->plans.push_back(p);
  }
  int st = batch_build(b);
  if (st == ST_OK) st = batch_capture(b);
  if (st != ST_OK) {
    batch_free(b);
    delete b;
    return st;
  }
  *batch = reinterpret_cast<hptt_cuda_batch_t>(b);
  return HPTT_OK;
}

int hptt_cuda_batch_refresh(hptt_cuda_batch_t batch) {
  Batch *b = reinterpret_cast<Batch *>(batch);
  if (!batch_valid(b)) return HPTT_ERR_HANDLE;
  return batch_build(b);
}

int hptt_cuda_batch_exec(hptt_cuda_batch_t batch, void *stream) {
  Batch *b = reinterpret_cast<Batch *>(batch);
  if (!batch_valid(b)) return HPTT_ERR_HANDLE;
  return batch_enqueue(b, static_cast<cudaStream_t>(stream));
}

int hptt_cuda_batch_info(hptt_cuda_batch_t batch, uint64_t *bytes, uint32_t *work_items,
                         uint32_t *kernels) {
  Batch *b = reinterpret_cast<Batch *>(batch);
  if (!batch_valid(b)) return HPTT_ERR_HANDLE;
  if (bytes) *bytes = b->bytes;
  if (work_items) *work_items = static_cast<uint32_t>(b->work.size());
  if (kernels) *kernels = static_cast<uint32_t>(b->groups.size());
  return HPTT_OK;
}

int hptt_cuda_batch_destroy(hptt_cuda_batch_t batch) {
  Batch *b = reinterpret_cast<Batch *>(batch);
  if (!batch_valid(b)) return HPTT_ERR_HANDLE;
  batch_free(b);
  b->magic = 0;
  delete b;
  return HPTT_OK;
}

int hptt_cuda_plan_exec_many(const hptt_cuda_plan_t *plans, uint32_t count, void *stream) {
  if (count && !plans) return HPTT_ERR_HANDLE;
  for (uint32_t i = 0; i < count; ++i) {
    Plan *p = reinterpret_cast<Plan *>(plans[i]);
    if (!plan_valid(p)) return HPTT_ERR_HANDLE;
    const int st = plan_enqueue(p, static_cast<cudaStream_t>(stream));
    if (st != ST_OK) return st;
  }
  return HPTT_OK;
}

}  // extern "C"
