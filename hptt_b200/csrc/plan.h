// Plan object behind the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "desc.h"
#include "planner.h"

namespace hptt_b200 {

constexpr uint32_t kPlanMagic = 0x48505454u;  // "HPTT"

struct Plan {
  uint32_t magic = kPlanMagic;
  HpttArgs args{};          // fused problem, vector tile, scalars, pointers
  HpttTile tile_scalar{};   // same problem without vector accesses
  int vec = 1;              // planned elements per access (KIND_ROWS)
  int grid = 0, grid_scalar = 0;
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  uint64_t elements = 0;    // N = prod(in_size)
  TileParams params;        // chosen by heuristic or tuner
  bool tuned = false;
  void *dtab = nullptr;         // device offset tables for args.t
  void *dtab_scalar = nullptr;  // ... and for tile_scalar (may alias dtab)
  // the tile the batch kernels (256 threads per CTA) run: args.t / dtab
  // when that has 256 threads, else the same parameters planned for 256
  HpttTile tile_batch{};
  void *dtab_batch = nullptr;
};

// Threads per CTA of the batch kernels.
constexpr int kBatchThreads = 256;

// Release the plan's device tables.
void plan_free_tables(Plan *p);

// Fill scalars/mode/update from alpha, beta.
void set_scalars(HpttArgs *a, const double *alpha, const double *beta,
                 int complex_scalars);

// Plan the tile for `params` and size the grid.  Needs a current device.
int plan_tiles(Plan *p, const TileParams &params);

// Enqueue one exec of the plan on `stream`.
int plan_enqueue(Plan *p, cudaStream_t stream);

// Same, with other data pointers (the plan is not modified).
int plan_enqueue_with(const Plan *p, const void *A, void *B, cudaStream_t stream);

// The effective vector width and tile for the current pointers.
int plan_vec_for_ptrs(const Plan *p);

bool plan_valid(const Plan *p);

}  // namespace hptt_b200
