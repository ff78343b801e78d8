// Tile-shape autotuner with a per-(dtype, rank, perm, size class, extent
// classes) cache.
//
// Replaces the reference's timing tuner PlanTrans::tuning_
// (inc/hptt/plan/plan_trans.tcc:33-67).  The reference times its candidates
// on the caller's buffers with alpha = 0, beta = 1, which rewrites B (-0
// becomes +0, and a non-finite A poisons B); this tuner reads A and writes
// only a scratch buffer of B's footprint.
#pragma once

#include <string>

#include "plan.h"
#include "planner.h"

namespace hptt_b200 {

// Time candidate tile parameters for `p` (its problem, scalars and A
// pointer) and return the fastest.  timeout < 0: every candidate; > 0: stop
// after that many seconds.  The winner is stored in the cache.
int autotune(Plan *p, double timeout, TileParams *best);

// Cached parameters for this plan's key, if any.
bool autotune_cache_lookup(const Plan *p, TileParams *out);

// Cache key text (GPU, dtype, fused rank, fused perm, size class, B read,
// extent class of every fused dim).
std::string autotune_key(const Plan *p);

// Load/save the cache file named by HPTT_B200_TUNE_CACHE (no-op if unset)
// or by `path` when given.
int autotune_cache_load(const char *path);
int autotune_cache_save(const char *path);
void autotune_cache_clear();
int autotune_cache_size();

}  // namespace hptt_b200
