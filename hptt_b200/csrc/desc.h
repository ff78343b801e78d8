// Problem and tile descriptors shared by the host planner and the sm_100a
// kernels.  Plain-old-data: passed to kernels by value (single transpose) or
// stored in a device table (batched / served forms).
#pragma once

#include <stdint.h>

#define HPTT_MAX_RANK 8

// Element kinds (same numbering as include/hptt_cuda.h).
enum HpttDtype : int32_t { DT_F32 = 0, DT_F64 = 1, DT_C64 = 2, DT_C128 = 3 };

// Arithmetic modes.
//   MODE_COPY   alpha == 1 exactly and B not updated: out = a (bit copy; equal
//               to fl(1*a) for every non-NaN a, and keeps NaN payloads as the
//               reference's x86 multiply does for quiet NaNs).
//   MODE_REAL   real scalars; complex types are scaled per component
//               (reference semantics, inc/hptt/types.h:29-54).
//   MODE_CPLX   complex scalars for complex types (extension).
enum HpttMode : int32_t { MODE_COPY = 0, MODE_REAL = 1, MODE_CPLX = 2 };

// Kernel kinds.
//   KIND_TILE  tiles pair input-contiguous dims (X) with output-contiguous
//              dims (Y) and go through shared memory.
//   KIND_ROWS  the fused stride-1 dimension is shared by A and B: rows are
//              copied/scaled directly, no shared-memory transpose.
//   KIND_VTILE tiles whose X side is one contiguous run of A and whose Y side
//              is one contiguous run of B, moved as 16-byte vectors (see
//              vtile.cuh); elements of at most 8 bytes.
//   KIND_TTILE tiles of boxes loaded and stored by the tensor memory
//              accelerator (see ttile.cuh); fused rank <= 5, 4- or 8-byte
//              elements, strides other than the unit one multiples of 16 bytes.
enum HpttKind : int32_t { KIND_TILE = 0, KIND_ROWS = 1, KIND_VTILE = 2, KIND_TTILE = 3 };

// Fused problem.  Dimensions are listed in INPUT order; sA/sB are the strides
// (in elements) of input dim d in A and in B.  perm[k] = input dim that is
// output dim k.
struct HpttProblem {
  int32_t dtype;
  int32_t rank;
  int64_t n[HPTT_MAX_RANK];
  int64_t sA[HPTT_MAX_RANK];
  int64_t sB[HPTT_MAX_RANK];
  int32_t perm[HPTT_MAX_RANK];
};

// A thread's slots q = q0 + j * R along a tile side with exactly two dims,
// walked without the side's offset table: q = d0 + e0 * d1 with offset
// d0 * s0 + d1 * s1, and a step of R adds r0 = R % e0 to d0 (one carry at
// most) and step = r0 * s0 + (R / e0) * s1 to the offset; a carry adds
// carry = s1 - e0 * s0.  e0 == 0: the side is not walked (one dim, three or
// more, or offsets beyond 32 bits).  mul/shr: fast division by e0.
struct HpttWalk {
  int32_t e0, r0, step, carry, s0, s1;
  uint32_t mul;
  int32_t shr;
};

// Tile shape and grid decomposition.
//
// A tile is W x X x Y elements:
//   W  the shared stride-1 block (input dim 0 when it is also output dim 0,
//      else W = 1),
//   X  input-side dims (input order) after W; all full except the last
//      (xc, tile extent xt[nx-1]),
//   Y  output-side dims (output order) after W; all full except the last
//      (yc).
// Load phase: element (w, x, y) -> e = w + W*x (RW = W*TX), row y.
// Store phase: e2 = w + W*y (WTY = W*TY), column x.
// Shared memory keeps element (w, x, y) at y*LD + e.
// KIND_ROWS uses W = the row chunk (vector lanes), X empty, Y = other dims.
struct HpttTile {
  int32_t kind;
  int32_t nt;        // threads per CTA
  int32_t vec;       // elements per vector access (KIND_ROWS only)
  int32_t W;
  int32_t nx, ny;
  int32_t xd[HPTT_MAX_RANK], xt[HPTT_MAX_RANK];
  int32_t yd[HPTT_MAX_RANK], yt[HPTT_MAX_RANK];
  int32_t TX, TY, RW, WTY, LD;
  int32_t R1, J1, R2, J2;     // threads-per-pass mapping, iterations
  int32_t xc, yc;             // chunked input dims, -1 when none
  int32_t wc;                 // chunked W dim (KIND_ROWS), -1 when none
  // grid: tile index -> origin.  gd = input dim, gcnt = number of positions,
  // gstep = tile extent along that dim (1 for dims outside the tile).
  int32_t px, py;             // extent products of the full X (Y) dims before
                              // the chunked last one: x = rest + px * c_last
  int32_t ng;
  int32_t gd[HPTT_MAX_RANK];
  uint32_t gcnt[HPTT_MAX_RANK];
  uint32_t gmul[HPTT_MAX_RANK];  // fast division by gcnt: q = umulhi(n, gmul) >> gshr
  int32_t gshr[HPTT_MAX_RANK];   // (gmul = 0 encodes gcnt == 1)
  int32_t gstep[HPTT_MAX_RANK];
  // per grid level, folded for the device (static-offset parameter reads):
  // the origin advances by c * gsa[g] in A and c * gsb[g] in B; gn = extent
  // of dim gd[g]; gflag bit 0 / 1: gd[g] is the chunked X / Y dim (xc / yc,
  // for KIND_ROWS wc / yc)
  int64_t gsa[HPTT_MAX_RANK], gsb[HPTT_MAX_RANK];
  int64_t gn[HPTT_MAX_RANK];
  int32_t gflag[HPTT_MAX_RANK];
  // single-dim sides: strides of the X dim in A and B, of the Y dim in A
  // and B (0 when that side has no dim or several)
  int64_t sxa, sxb, sya, syb;
  uint32_t num_tiles;
  int32_t big_offsets;        // 1 when in-tile offsets need 64 bits
  int32_t smem_bytes;         // dynamic shared memory for one CTA
  // Byte offsets inside the plan's device table buffer (HpttArgs::tables).
  // KIND_TILE:
  //   [0]         TY x HpttTabEnt: row slot q -> {A offset of the row, its
  //               coordinate along the chunked Y dim}; slots enumerate the Y
  //               dims in INPUT order, so consecutive slots are adjacent in A
  //   [tab2_off]  TX x HpttTabEnt: column slot q -> {B offset of the column,
  //               its coordinate along the chunked X dim}; slots enumerate the
  //               X dims in OUTPUT order, so consecutive slots are adjacent in B
  //   [thr_off]   nt x HpttThr per-thread constants
  // KIND_ROWS: A row offsets (TY x OffT) at 0, B row offsets at tab2_off.
  // KIND_VTILE: TY x OffT at 0, row y (Y dims in output order) -> A offset
  // of the row; TX x OffT at tab2_off, column x (X dims in input order) ->
  // B offset of the column.
  int32_t tab2_off, thr_off, table_bytes;
  // fast division by R1 and R2 (same scheme as gmul/gshr)
  uint32_t r1_mul, r2_mul;
  int32_t r1_shr, r2_shr;
  // KIND_TILE: 1 when TY == R1 * J1 and TX == R2 * J2, so in a tile that
  // lies wholly inside the tensor every loading thread has exactly J1 rows
  // and every storing thread J2 columns
  int32_t even;
  // tile extent along the chunked X / Y dim (1 when that side is not
  // chunked): a tile with remX >= xce and remY >= yce lies wholly inside
  int32_t xce, yce;
  // fast division by TX and TY: per-thread constants of single-dim tiles
  // with W == 1 are computed from threadIdx instead of read from the table
  uint32_t tx_mul, ty_mul;
  int32_t tx_shr, ty_shr;
  // update tiles with single-dim sides: 1 = interior tiles run exact trip
  // counts (tile_table_interior_k), 0 = the general predicated path
  int32_t upd_exact;
  // two-dim sides: the X side's column slots (B offsets, step R2) and the Y
  // side's row slots (A offsets, step R1)
  HpttWalk wx, wy;
  // KIND_VTILE: log2 of the 8-slot groups along a row of the load phase
  // (vlx) and along a column of the store phase (vly); a row has 8 << vlx
  // vector slots, a column 8 << vly; vj = the most 16-byte vectors a thread
  // holds per phase (4 or 8: two kernel builds with their own register
  // budgets); vpre = 1: an update tile of the four-vector build reads its B
  // windows before its A loads
  int32_t vlx, vly, vj, vpre;
  // KIND_TTILE: boxes per tile along input dim 0 (tkx) and along the output's
  // leading dim (tky); ts = 0: one CTA per tile, 2-4: persistent CTAs that
  // keep ts tiles of loads in flight (a ring of ts stages)
  int32_t tkx, tky, ts;
};

// One slot of a KIND_TILE offset table (OffT = uint32_t or int64_t).
template <typename OffT>
struct alignas(sizeof(OffT) * 2) HpttTabEnt {
  OffT off;
  int32_t c;  // coordinate along the chunked dim (0 when none is chunked)
};

// Per-thread constants of the tile transpose, precomputed on the host.
// Load phase: the thread owns element e (= w + W*x) of every row slot
// q0 + j*R1; store phase: element e2 (= w + W*y) of every column slot
// qs0 + j*R2.
struct alignas(16) HpttThr {
  int64_t inE;     // A offset of element e
  int64_t outE2;   // B offset of element e2
  int32_t q0, qs0; // first row slot (load), first column slot (store)
  int32_t sme;     // shared-memory column of element e: qcol(x) * W + w
  int32_t sme2;    // shared-memory row start of element e2: qrow(y) * LD + w
  int32_t cxe;     // coordinate of e along the chunked X dim (0 if none)
  int32_t cye2;    // coordinate of e2 along the chunked Y dim (0 if none)
  int32_t active;  // bit 0: loads, bit 1: stores
  int32_t pad;
};

// Per-thread iterations of one phase, sized so every thread keeps about 64
// (tile) or 128 (rows) bytes of loads in flight without spilling.  (A tile
// that also reads B keeps twice that: its B values are loaded alongside.)
#ifdef __CUDACC__
#define HPTT_HD __host__ __device__
#else
#define HPTT_HD
#endif
HPTT_HD constexpr int hptt_jmax_tile(int elem_bytes) {
  return elem_bytes >= 16 ? 4 : (elem_bytes >= 8 ? 8 : 16);
}
HPTT_HD constexpr int hptt_jmax_rows(int access_bytes) {
  return access_bytes >= 16 ? 4 : (access_bytes >= 8 ? 8 : 16);
}


// Everything one launch (or one batch entry) needs.
struct HpttArgs {
  HpttProblem p;
  HpttTile t;
  const void *A;
  void *B;
  const void *tables;  // device buffer laid out as HpttTile::tab2_off/thr_off say
  double alpha[2];
  double beta[2];
  int32_t mode;
  int32_t update;
};
