// Per-plan offset tables (host side).
#pragma once

#include <vector>

#include "desc.h"

namespace hptt_b200 {

// Fill `out` (T.table_bytes bytes) with the tables the kernels read:
// KIND_TILE: row offsets in A, column offsets in B, per-thread constants;
// KIND_ROWS: row offsets in A and in B.  Offsets are 32- or 64-bit as
// T.big_offsets says.
void build_tables(const HpttProblem &P, const HpttTile &T, std::vector<unsigned char> *out);

}  // namespace hptt_b200
