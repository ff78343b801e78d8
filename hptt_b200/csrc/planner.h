// Host planner: argument guard, index fusion and tile/grid selection.
#pragma once

#include <stdint.h>
#include <string>
#include <vector>

#include "desc.h"

namespace hptt_b200 {

// Status codes (mirrored in include/hptt_cuda.h).
enum Status : int {
  ST_OK = 0,
  ST_NULL_DATA = 1,        // in or out pointer is null
  ST_BAD_RANK = 2,         // rank < 2 (or above the supported maximum)
  ST_BAD_SIZE_VECTOR = 3,  // a size vector has the wrong length
  ST_BAD_SIZE_VALUE = 4,   // zero extent or outer size below inner size
  ST_BAD_PERM = 5,         // perm is not a permutation
  ST_BAD_DTYPE = 6,
  ST_CUDA = 7,             // a CUDA runtime call failed
  ST_NO_DEVICE = 8,
  ST_ALLOC = 9,            // host or device allocation failed
  ST_BUDGET = 10,          // request exceeds the memory budget
  ST_BAD_HANDLE = 11,      // null or destroyed plan/batch/server
  ST_TIMEOUT = 12,         // a bounded wait ran out
  ST_TOO_LARGE = 13,       // a size beyond what this build supports
  ST_BUSY = 14,            // no free slot (served form)
  ST_LABELS = 15,          // contraction labels do not describe a contraction
  ST_BLAS = 16,            // a cuBLAS call failed (contraction GEMM)
};

const char *status_string(int st);

// Tuning knobs of the tile chooser; the autotuner searches over these.
struct TileParams {
  int nt = 256;            // threads per CTA
  int run_bytes = 256;     // contiguous bytes wanted on each side of a tile
  int vmin_bytes = 16384;  // grow tiles to at least this many bytes
  int smem_bytes = 32768;  // data bytes one tile may hold in shared memory
  int rows_min_bytes = 512;  // shared stride-1 run long enough for KIND_ROWS
  int ctas_per_sm = 0;     // 0: as many as fit
  int max_vec_bytes = 16;  // widest vector access (KIND_ROWS)
  int y_first = 0;         // choose the output-side dims before the input side
  int max_iters = 0;       // cap on per-thread iterations of a tile (0: the
                           // kernel's own limit, hptt_jmax_tile)
  int full_side = 0;       // single-dim tiles: 1 = take the whole X extent,
                           // 2 = the whole Y extent, shrinking the other side
                           // (short rows that are not sector-aligned then
                           // become one contiguous range per tile)
  int walk = 1;            // two-dim tile sides: walk the slot offsets (1) or
                           // read the side's table (0); HpttWalk
  int upd_exact = 1;       // update tiles with single-dim sides: exact trip
                           // counts in interior tiles (1) or the general
                           // predicated path (0); HpttTile::upd_exact
  int grid_order = 0;      // grid levels after the chunked tile dims: in
                           // input order (0), or by the smaller of each
                           // dim's A and B strides (1), so tiles that share
                           // partially written sectors run close in time
  int vt = 0;              // 1: a vector tile (KIND_VTILE) where the shape
                           // allows one, else the tile above
  int vt_nvx = 16;         // vector slots along a row (load) and along a
  int vt_nvy = 16;         // column (store) of a vector tile: 8, 16 or 32
  int vt_j = 8;            // 16-byte vectors a vector-tile thread holds per
                           // phase: 8 (64 registers) or 4 (32 registers)
  int vt_pre = 0;          // 1: update tiles with vt_j == 4 read B before A
                           // (64 registers)
  int tt = 0;              // a TMA tile (KIND_TTILE) where the shape allows
                           // one (takes precedence over vt): 1 = one CTA per
                           // tile, 2-4 = persistent CTAs with tt stages
  int tt_kx = 2;           // boxes per TMA tile along input dim 0 and along
  int tt_ky = 2;           // the output's leading dim (64 threads per box)
};

// Whether a TMA tile (KIND_TTILE) can serve this problem: fused rank 2-5,
// 4- or 8-byte elements, no shared stride-1 dim, every stride other than the
// unit one a multiple of 16 bytes and below 2^40 bytes, extents at most 2^30
// (box coordinates are signed 32-bit).
bool ttile_possible(const HpttProblem &p);

// The tensor map of one side of a KIND_TTILE tile: side 0 is A with its dims
// in input order, side 1 is B with its dims in output order.  stride_bytes[0]
// is the element size; box = the tile's box extents (1 outside the box).
struct TtileMapParams {
  int rank = 0;
  int elem_bytes = 0;
  uint64_t dims[5] = {0};
  uint64_t stride_bytes[5] = {0};
  uint32_t box[5] = {0};
};
int ttile_map_params(const HpttProblem &p, const HpttTile &t, int side, TtileMapParams *out);

// Whether a vector tile (KIND_VTILE) can serve this problem: elements of at
// most 8 bytes and no shared stride-1 dim.
bool vtile_possible(const HpttProblem &p);

// Reference argument guard (src/hptt.cc:25-56) plus the one check the
// reference omits for memory safety (out_outer[k] >= out_size[k]).
int validate(int rank, const uint32_t *in_size, const uint32_t *perm,
             const uint32_t *in_outer, const uint32_t *out_outer,
             int in_outer_len, int out_outer_len);

// Fuse index groups.  Output: problem in input-dim order with strides.
int fuse(int dtype, int rank, const uint32_t *in_size, const uint32_t *perm,
         const uint32_t *in_outer, const uint32_t *out_outer,
         HpttProblem *out);

// Choose tile and grid.  Returns ST_OK or ST_TOO_LARGE.
// `update` != 0 when B is read (its tile is staged in shared memory too).
int choose_tile(const HpttProblem &p, const TileParams &tp, int update, HpttTile *t);

int elem_bytes(int dtype);

// Host-side index maps of a KIND_TILE tile.  Row slots enumerate the Y dims
// in INPUT order (consecutive slots are adjacent in A); column slots
// enumerate the X dims in OUTPUT order (consecutive slots are adjacent in B).
struct TileMaps {
  std::vector<int> qrow;      // row index y (Y order) -> row slot
  std::vector<int> qcol;      // column index x (X order) -> column slot
  std::vector<int64_t> offA;  // row slot -> A offset
  std::vector<int> cy;        // row slot -> coordinate along the chunked Y dim
  std::vector<int64_t> offB;  // column slot -> B offset
  std::vector<int> cx;        // column slot -> coordinate along the chunked X dim
};
void tile_maps(const HpttProblem &p, const HpttTile &t, TileMaps *m);

// Host-side index maps of a KIND_VTILE tile: rowA[y] = A offset of row y
// (the Y dims in output order), colB[x] = B offset of column x (the X dims in
// input order).
void vtile_maps(const HpttProblem &p, const HpttTile &t, std::vector<int64_t> *rowA,
                std::vector<int64_t> *colB);

// Per-thread constants of thread `tid` (uses t.LD).
HpttThr tile_thread_consts(const HpttProblem &p, const HpttTile &t, const TileMaps &m, int tid);

// Human-readable plan summary (print_plan()).
std::string describe(const HpttProblem &p, const HpttTile &t);

}  // namespace hptt_b200
