// Batched form: many independent transposes in one graph launch.
//
// Each entry of a batch is a snapshot of a plan's launch arguments (fused
// problem, tuned tile, device offset tables, data pointers, scalars) in a
// device descriptor table.  A work list splits every entry's tiles into
// items of at most kBatchChunkMax tiles, sorted into groups by tile body
// (element storage, arithmetic, B read, tile shape).  Each group has its own
// persistent kernel -- specialised like the single-transpose kernel of that
// body -- whose CTAs take the group's items from an atomic counter.  One CUDA
// graph holds a counter reset and all group kernels as independent nodes, so
// the groups run side by side on the device and one graph launch runs the
// whole batch.  Every result is bit-identical to the entry's own exec.
// Descriptors, work list and counters live in device memory: refreshing the
// entries' pointers or scalars keeps the graph unless the launch shape
// changes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "desc.h"

namespace hptt_b200 {

constexpr uint32_t kBatchMagic = 0x48505442u;  // "HPTB"
constexpr uint32_t kBatchChunkMax = 16;

// One descriptor: the launch arguments and the tile body that runs them.
struct alignas(16) HpttBatchDesc {
  HpttArgs a;
  int32_t body;  // combo * kBatchShapes + shape, see batch.cu
  int32_t vec;
  int32_t pad[2];
};

// A run of tiles of one descriptor.
struct alignas(16) HpttWork {
  uint32_t desc, tile0, ntiles, pad;
};

struct Plan;

// One group: the items [begin, end) of the work list, all of one body.
struct BatchGroup {
  int body = 0;
  uint32_t begin = 0, end = 0;
  int smem_bytes = 0;
  int grid = 0;
};

struct Batch {
  uint32_t magic = kBatchMagic;
  int device = 0;
  std::vector<Plan *> plans;          // not owned; must outlive the batch
  std::vector<HpttBatchDesc> desc;    // host copy of the descriptor table
  std::vector<HpttWork> work;         // host copy of the work list
  HpttBatchDesc *d_desc = nullptr;
  HpttWork *d_work = nullptr;
  uint32_t work_capacity = 0;
  std::vector<BatchGroup> groups;
  uint32_t *d_counters = nullptr;     // one item counter per group
  uint32_t counter_capacity = 0;
  uint64_t bytes = 0;                 // algorithmic bytes of one exec
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
};

bool batch_valid(const Batch *b);

// One entry to lay out: a plan, optionally with other data pointers (both
// null: the plan's own).
struct BatchEntry {
  const Plan *plan = nullptr;
  const void *A = nullptr;
  void *B = nullptr;
};

// Descriptors, grouped work list and group launch shapes for a set of
// entries on the current device (sms = its multiprocessor count).
struct BatchLayout {
  std::vector<HpttBatchDesc> desc;
  std::vector<HpttWork> work;
  std::vector<BatchGroup> groups;
  uint64_t bytes = 0;
};
int batch_layout(const std::vector<BatchEntry> &entries, int sms, BatchLayout *layout);

// Launch one group kernel (its counter must be zero).
int batch_launch_group(const BatchGroup &g, const HpttBatchDesc *d_desc, const HpttWork *d_work,
                       uint32_t *d_counter, cudaStream_t stream);

// Reset the group counters and launch every group kernel on `stream` (one
// after another), reading descriptors and work items from device memory.
int batch_launch_groups(const std::vector<BatchGroup> &groups, const HpttBatchDesc *d_desc,
                        const HpttWork *d_work, uint32_t *d_counters, cudaStream_t stream);

// Build descriptors and the work list for the plans' current pointers and
// upload them (allocating device memory on first use).
int batch_build(Batch *b);

// Enqueue one exec: the graph when there is one, else the counter reset
// and the group kernels one after another on `stream`.
int batch_enqueue(Batch *b, cudaStream_t stream);

// Build the CUDA graph (counter reset -> every group kernel), replacing any.
int batch_capture(Batch *b);

void batch_free(Batch *b);

}  // namespace hptt_b200
