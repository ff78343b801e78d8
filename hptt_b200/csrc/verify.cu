// Host emulation of the kernels' addressing, for CPU tests.
//
// Runs the planner, builds the same offset tables a plan uploads, then
// replays every CTA (one per tile) and every thread of the launch exactly as
// tile_one / rows_one in kernels.cuh index memory, and checks, without a GPU:
//   - every A read and every B read/write is inside the caller's buffers,
//   - every shared-memory access is inside the tile buffer and reads a slot
//     the load phase of the same tile wrote,
//   - the element stored to B[j] is the one loaded from A[i] with
//     j = perm-mapped(i), and every inner element of B is written exactly
//     once while the padding of B is never touched.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/hptt_cuda.h"
#include "kernels.cuh"
#include "planner.h"
#include "tables.h"
#include "ttile.cuh"
#include "vtile.cuh"

namespace hptt_b200 {
namespace {

using namespace dev;

struct Layout {
  int rank;
  std::vector<int64_t> in_size, in_outer, out_outer, perm;
  int64_t nA = 1, nB = 1;
  std::vector<int64_t> sbo;  // output strides per output dim
};

// A index -> expected B index, or -1 if the A index is padding.
int64_t map_a_to_b(const Layout &L, int64_t ia) {
  int64_t c[HPTT_MAX_RANK];
  int64_t rem = ia;
  for (int d = 0; d < L.rank; ++d) {
    c[d] = rem % L.in_outer[d];
    rem /= L.in_outer[d];
    if (c[d] >= L.in_size[d]) return -1;
  }
  int64_t ib = 0;
  for (int k = 0; k < L.rank; ++k) ib += c[L.perm[k]] * L.sbo[k];
  return ib;
}

bool b_is_inner(const Layout &L, int64_t ib) {
  int64_t rem = ib;
  for (int k = 0; k < L.rank; ++k) {
    const int64_t c = rem % L.out_outer[k];
    rem /= L.out_outer[k];
    if (c >= L.in_size[L.perm[k]]) return false;
  }
  return true;
}

// fast: replay the single-transpose kernel (tile_one with FAST); else the
// persistent batch kernels (FAST off: no update fast forms, clamped
// table-driven interiors, no walked sides).
template <typename OffT>
int replay_tile(const HpttProblem &P, const HpttTile &T, int update, const Layout &L,
                const std::vector<unsigned char> &tab, std::vector<uint8_t> &writes,
                uint64_t *checked, bool fast) {
  const int esz = elem_bytes(P.dtype);
  const int J = hptt_jmax_tile(esz);
  (void)update;
  if (T.J1 > J || T.J2 > J) return 101;
  if (T.smem_bytes < T.TY * T.LD * esz) return 102;
  using Ent = HpttTabEnt<OffT>;
  if (T.tab2_off < T.TY * static_cast<int>(sizeof(Ent))) return 103;
  if (T.thr_off < T.tab2_off + T.TX * static_cast<int>(sizeof(Ent))) return 104;
  if (T.table_bytes < T.thr_off + T.nt * static_cast<int>(sizeof(HpttThr))) return 105;
  if (T.thr_off % 16 || T.tab2_off % 16) return 106;
  const Ent *tabY = reinterpret_cast<const Ent *>(tab.data());
  const Ent *tabX = reinterpret_cast<const Ent *>(tab.data() + T.tab2_off);
  const HpttThr *thr = reinterpret_cast<const HpttThr *>(tab.data() + T.thr_off);
  // Single-dim sides skip the tables in the kernel (offset q * stride,
  // coordinate q along the chunked dim): the tables must hold exactly that,
  // so replaying the tables replays those kernels too.
  if (T.ny <= 1) {
    const int64_t sY = T.ny == 1 ? P.sA[T.yd[0]] : 0;
    for (int q = 0; q < T.TY; ++q)
      if (static_cast<int64_t>(tabY[q].off) != q * sY || tabY[q].c != (T.yc >= 0 ? q : 0))
        return 119;
  }
  if (T.nx <= 1) {
    const int64_t sX = T.nx == 1 ? P.sB[T.xd[0]] : 0;
    for (int q = 0; q < T.TX; ++q)
      if (static_cast<int64_t>(tabX[q].off) != q * sX || tabX[q].c != (T.xc >= 0 ? q : 0))
        return 120;
  }
  // single-dim sides with W == 1: the kernel computes the per-thread
  // constants from the thread index; they must equal the table's
  if (!T.big_offsets && T.nx == 1 && T.ny == 1 && T.W == 1) {
    for (int t = 0; t < T.nt; ++t) {
      const HpttThr a = thread_consts_1d(P, T, t), &b = thr[t];
      if (a.q0 != b.q0 || a.qs0 != b.qs0 || a.inE != b.inE || a.outE2 != b.outE2 ||
          a.sme != b.sme || a.sme2 != b.sme2 || a.cxe != b.cxe || a.cye2 != b.cye2 ||
          a.active != b.active)
        return 131;
    }
  }
  const int64_t smem_elems = static_cast<int64_t>(T.TY) * T.LD;
  std::vector<int64_t> slot(smem_elems);
  // the kernel's single-dim-side variants (kernels.cu: pick_tile)
  const bool ly = !T.big_offsets && T.ny <= 1, lx = !T.big_offsets && T.nx <= 1;
  // the interior fast path (kernels.cuh) assumes every loading thread has
  // J1 rows and every storing thread J2 columns
  if (T.even && !(T.TY == T.R1 * T.J1 && T.TX == T.R2 * T.J2)) return 130;
  // the kernel indexes single-dim sides as q * stride in 32-bit ints
  if (ly && T.ny == 1 && T.TY > 1 && P.sA[T.yd[0]] > 0x7fffffffLL) return 128;
  if (lx && T.nx == 1 && T.TX > 1 && P.sB[T.xd[0]] > 0x7fffffffLL) return 129;
  // tiles with single-dim sides run compile-time loops (copy/scale tiles
  // always, update tiles of 8/16-byte elements when J1 == J2 == J): interior
  // tiles of even shapes
  // unclamped, every other tile with slot indices clamped to the last valid
  // row/column (kernels.cuh: tile_clamped, tile_full_upd), so an iteration
  // past the edge repeats a slot with the same element
  const bool clamped_kind =
      lx && ly && (!update || (fast && T.J1 == J && T.J2 == J && elem_bytes(P.dtype) > 4));
  // tiles with a multi-dim side, interior tiles.  Single-transpose kernel
  // (kernels.cuh: tile_table_interior_k): copy, scale and update tiles run
  // exact trip counts, a thread's last slot alone tested against the side's
  // end, offsets from the tables, from q * stride (one dim) or from a walk
  // (two dims, HpttWalk -- replayed here against the tables).  Batch kernels
  // (tile_table_interior_clamped): copy/scale tiles only, every slot past
  // the end clamped to the last one.
  const bool table_kind = fast && (!(lx && ly) || (update && T.upd_exact));
  const bool table_clamped_kind = !fast && !update && !(lx && ly);
  const bool tracks = clamped_kind || table_clamped_kind;
  // walked sides: the walk must give the table's offset at every slot a
  // thread reaches (kernels.cuh: walk_start / walk_step)
  if (fast && !T.big_offsets) {
    for (int side = 0; side < 2; ++side) {
      const HpttWalk &w = side ? T.wx : T.wy;
      if (w.e0 == 0) continue;
      if ((side ? T.nx : T.ny) != 2) return 154;
      const int R = side ? T.R2 : T.R1, N = side ? T.J2 : T.J1, lim = side ? T.TX : T.TY;
      const Ent *tb = side ? tabX : tabY;
      for (int q0 = 0; q0 < R; ++q0) {
        WalkPos wp = walk_start(w, q0);
        for (int j = 0; j < N; ++j) {
          const int q = q0 + j * R;
          if (q < lim && wp.off != static_cast<uint32_t>(tb[q].off)) return 155;
          walk_step(w, wp);
        }
      }
    }
  }
  std::vector<int64_t> writer(tracks ? static_cast<size_t>(L.nB) : 0, -1);
  std::vector<uint32_t> writer_tile(tracks ? static_cast<size_t>(L.nB) : 0, 0);
  for (uint32_t tile = 0; tile < T.num_tiles; ++tile) {
    const TileOrigin o = tile_origin(P, T, tile);
    std::fill(slot.begin(), slot.end(), -1);
    const int limQY = (ly && T.yc >= 0 && o.remY < T.TY) ? o.remY : T.TY;
    const int limQX = (lx && T.xc >= 0 && o.remX < T.TX) ? o.remX : T.TX;
    const bool interior = T.even && o.remX >= T.TX && o.remY >= T.TY;
    const bool inside = o.remX >= T.xce && o.remY >= T.yce;
    // update tiles with single-dim sides that tile_interior_upd or
    // tile_full_upd take first (kernels.cuh: tile_one)
    const bool upd_fast_form = update && fast && lx && ly && T.J1 == J && T.J2 == J &&
                               ((T.even && interior) || esz > 4);
    if (table_kind && inside && !upd_fast_form) {
      // predicated exact-trip-count form: every slot once
      for (int t = 0; t < T.nt; ++t) {
        const HpttThr &th = thr[t];
        if (!(th.active & 1)) continue;
        for (int j = 0; j < T.J1; ++j) {
          const int q = th.q0 + j * T.R1;
          if (q >= T.TY) {
            if (j != T.J1 - 1) return 156;  // only the last iteration may pass the end
            continue;
          }
          if (!(tabY[q].c < o.remY) || th.cxe >= o.remX) return 157;
          const int64_t si = static_cast<int64_t>(q) * T.LD + th.sme;
          if (si < 0 || si >= smem_elems) return 158;
          if (slot[si] >= 0) return 159;  // two writers of one slot
          const int64_t ia = o.bA + th.inE + static_cast<int64_t>(tabY[q].off);
          if (ia < 0 || ia >= L.nA) return 160;
          slot[si] = ia;
        }
      }
      for (int t = 0; t < T.nt; ++t) {
        const HpttThr &th = thr[t];
        if (!(th.active & 2)) continue;
        for (int j = 0; j < T.J2; ++j) {
          const int q = th.qs0 + j * T.R2;
          if (q >= T.TX) {
            if (j != T.J2 - 1) return 161;
            continue;
          }
          if (!(tabX[q].c < o.remX) || th.cye2 >= o.remY) return 162;
          const int64_t si = static_cast<int64_t>(th.sme2) + static_cast<int64_t>(q) * T.W;
          if (si < 0 || si >= smem_elems) return 163;
          const int64_t ia = slot[si];
          if (ia < 0) return 164;  // reads a slot no load wrote
          const int64_t ib = o.bB + th.outE2 + static_cast<int64_t>(tabX[q].off);
          if (ib < 0 || ib >= L.nB) return 165;
          if (map_a_to_b(L, ia) != ib) return 166;
          if (writes[ib] != 0) return 167;  // one write per element (B read once too)
          writes[ib] = 1;
          ++*checked;
        }
      }
      continue;
    }
    const bool table_interior = table_clamped_kind && inside;
    if ((clamped_kind && !interior) || table_interior) {
      const int limR = table_interior ? T.TY : (T.yc >= 0 && o.remY < T.TY) ? o.remY : T.TY;
      const int limC = table_interior ? T.TX : (T.xc >= 0 && o.remX < T.TX) ? o.remX : T.TX;
      if (limR < 1 || limC < 1) return 140;
      for (int t = 0; t < T.nt; ++t) {
        const HpttThr &th = thr[t];
        if (!((th.active & 1) && th.cxe < o.remX)) continue;
        for (int j = 0; j < T.J1; ++j) {
          const int q = std::min(th.q0 + j * T.R1, limR - 1);
          if (q < 0 || q >= T.TY) return 141;
          if (!(tabY[q].c < o.remY)) return 142;
          const int64_t si = static_cast<int64_t>(q) * T.LD + th.sme;
          if (si < 0 || si >= smem_elems) return 143;
          const int64_t ia = o.bA + th.inE + static_cast<int64_t>(tabY[q].off);
          if (ia < 0 || ia >= L.nA) return 144;
          // a repeated slot must hold the same element
          if (slot[si] >= 0 && slot[si] != ia) return 145;
          slot[si] = ia;
        }
      }
      for (int t = 0; t < T.nt; ++t) {
        const HpttThr &th = thr[t];
        if (!((th.active & 2) && th.cye2 < o.remY)) continue;
        for (int j = 0; j < T.J2; ++j) {
          const int q = std::min(th.qs0 + j * T.R2, limC - 1);
          if (q < 0 || q >= T.TX) return 146;
          if (!(tabX[q].c < o.remX)) return 147;
          const int64_t si = static_cast<int64_t>(th.sme2) + static_cast<int64_t>(q) * T.W;
          if (si < 0 || si >= smem_elems) return 148;
          const int64_t ia = slot[si];
          if (ia < 0) return 149;  // reads a slot no load wrote
          const int64_t ib = o.bB + th.outE2 + static_cast<int64_t>(tabX[q].off);
          if (ib < 0 || ib >= L.nB) return 150;
          if (map_a_to_b(L, ia) != ib) return 151;
          // a repeated write must come from the same tile with the same element
          if (writer[ib] >= 0 && (writer[ib] != ia || writer_tile[ib] != tile)) return 152;
          if (writer[ib] < 0) {
            if (writes[ib] != 0) return 153;  // written by another tile
            writer[ib] = ia;
            writer_tile[ib] = tile;
            writes[ib] = 1;
            ++*checked;
          }
        }
      }
      continue;
    }
    // load phase: iteration j of a thread loads row slot q0 + j*R1 when
    // j < J1 and the slot is inside the tile (single-dim Y side: inside the
    // tensor too); a table slot outside the tensor re-reads element 0
    for (int t = 0; t < T.nt; ++t) {
      const HpttThr &th = thr[t];
      const bool ld_ok = (th.active & 1) && th.cxe < o.remX;
      if (!ld_ok) continue;
      for (int j = 0; j < J; ++j) {
        const int q = th.q0 + j * T.R1;
        if (!(j < T.J1 && q < (ly ? limQY : T.TY))) continue;
        if (q < 0 || q >= T.TY) return 125;
        if (ly && !(tabY[q].c < o.remY)) return 121;
        const int64_t si = static_cast<int64_t>(q) * T.LD + th.sme;
        if (si < 0 || si >= smem_elems) return 108;
        if (slot[si] >= 0 || slot[si] == -3) return 110;  // two writers of one slot
        if (tabY[q].c < o.remY) {
          const int64_t ia = o.bA + th.inE + static_cast<int64_t>(tabY[q].off);
          if (ia < 0 || ia >= L.nA) return 109;
          slot[si] = ia;
        } else {
          // the kernel re-reads this thread's first element of the tile
          const int64_t ia0 = o.bA + th.inE;
          if (ia0 < 0 || ia0 >= L.nA || map_a_to_b(L, ia0) < 0) return 117;
          slot[si] = -3;  // written, value unused
        }
      }
    }
    // store phase (and the B reads of the load phase, same addresses)
    for (int t = 0; t < T.nt; ++t) {
      const HpttThr &th = thr[t];
      const bool st_ok = (th.active & 2) && th.cye2 < o.remY;
      if (!st_ok) continue;
      for (int j = 0; j < J; ++j) {
        const int q = th.qs0 + j * T.R2;
        if (!(j < T.J2 && q < (lx ? limQX : T.TX))) continue;
        if (q < 0 || q >= T.TX) return 127;
        if (lx && !(tabX[q].c < o.remX)) return 122;
        if (!(tabX[q].c < o.remX)) {
          // the B prefetch re-reads this thread's first store element
          const int64_t ib0 = o.bB + th.outE2;
          if (ib0 < 0 || ib0 >= L.nB || !b_is_inner(L, ib0)) return 118;
          continue;
        }
        const int64_t si = static_cast<int64_t>(th.sme2) + static_cast<int64_t>(q) * T.W;
        if (si < 0 || si >= smem_elems) return 112;
        const int64_t ia = slot[si];
        if (ia < 0) return 113;  // reads a slot no valid load wrote
        const int64_t ib = o.bB + th.outE2 + static_cast<int64_t>(tabX[q].off);
        if (ib < 0 || ib >= L.nB) return 114;
        if (map_a_to_b(L, ia) != ib) return 115;
        if (writes[ib] != 0) return 116;
        writes[ib] = 1;
        ++*checked;
      }
    }
  }
  return 0;
}

// Vector tile (vtile.cuh: vtile_one), with the A and B base addresses
// `misA` / `misB` elements past a 16-byte boundary.  Every window the kernel
// reads must be 16-byte aligned and hold at least one element of its buffer
// (so it lies in the buffer's own 16-byte blocks); every 16-byte store must be
// aligned and wholly inside the column; every shared-memory access must stay
// inside the tile buffer, and the store phase must read, for each element it
// writes, the slot the load phase filled with the A element the permutation
// maps to it.
template <typename OffT>
int replay_vtile(const HpttProblem &P, const HpttTile &T, int update, const Layout &L,
                 const std::vector<unsigned char> &tab, std::vector<uint8_t> &writes,
                 uint64_t *checked, int misA, int misB) {
  const int esz = elem_bytes(P.dtype);
  const int V = 16 / esz, PD = V - 1;
  const int JV = T.vj;
  if (JV != 4 && JV != 8) return 300;
  if (V < 2) return 301;
  const int nvx = 8 << T.vlx, nvy = 8 << T.vly;
  const int GX = nvx / 8, GY = nvy / 8;  // slots of a line a thread takes
  // vectors a thread holds: J lines x slot groups, within the kernel's
  // compile-time limit
  if (T.J1 * GX > JV || T.J2 * GY > JV) return 302;
  if (T.R1 != T.nt / 8 || T.R2 != T.nt / 8) return 303;
  if (T.R1 * T.J1 < T.TY || T.R2 * T.J2 < T.TX) return 304;
  if (nvx * V - PD < T.TX || nvy * V - PD < T.TY) return 305;
  if (T.LD < nvx * V + PD) return 306;
  const int64_t rows = static_cast<int64_t>(nvy) * V + PD;
  if (T.smem_bytes < rows * T.LD * esz) return 307;
  if (T.tab2_off < T.TY * static_cast<int>(sizeof(OffT))) return 308;
  if (T.table_bytes < T.tab2_off + T.TX * static_cast<int>(sizeof(OffT))) return 309;
  const OffT *tabY = reinterpret_cast<const OffT *>(tab.data());
  const OffT *tabX = reinterpret_cast<const OffT *>(tab.data() + T.tab2_off);
  const bool ly = !T.big_offsets && T.ny <= 1, lx = !T.big_offsets && T.nx <= 1;
  // the kernel computes single-dim sides as q * stride in 32 bits: the
  // tables must hold exactly that
  for (int y = 0; y < T.TY; ++y) {
    const int64_t want = ly && T.ny == 1 ? static_cast<int64_t>(y) * T.sya : static_cast<int64_t>(tabY[y]);
    if (static_cast<int64_t>(tabY[y]) != want) return 310;
    if (ly && want > 0x7fffffffLL) return 311;
  }
  for (int x = 0; x < T.TX; ++x) {
    const int64_t want = lx && T.nx == 1 ? static_cast<int64_t>(x) * T.sxb : static_cast<int64_t>(tabX[x]);
    if (static_cast<int64_t>(tabX[x]) != want) return 312;
    if (lx && want > 0x7fffffffLL) return 313;
  }
  auto md = [V](int64_t v) { return static_cast<int>(((v % V) + V) % V); };
  const int64_t smem_elems = rows * T.LD;
  std::vector<int64_t> slot(static_cast<size_t>(smem_elems));
  // does [w, w + V) (elements from the buffer base) hold an element of [0, n)?
  auto window_ok = [V](int64_t w, int64_t n) { return w + V > 0 && w < n; };
  for (uint32_t tile = 0; tile < T.num_tiles; ++tile) {
    const TileOrigin o = tile_origin(P, T, tile);
    const int limX = vt_lim_x(T, o), limY = vt_lim_y(T, o);
    if (limX < 1 || limY < 1 || limX > T.TX || limY > T.TY) return 314;
    std::fill(slot.begin(), slot.end(), -1);
    for (int t = 0; t < T.nt; ++t) {
      const VtPos ps = vt_pos(t);
      if (ps.k >= 8 || ps.r0 >= T.R1) return 315;
      for (int j = 0; j < T.J1; ++j) {
        const int y = ps.r0 + j * T.R1;
        if (!(y < limY)) continue;
        const int64_t row = o.bA + static_cast<int64_t>(tabY[y]);  // element index in A
        const int sh = md(misA + row);
        for (int g = 0; g < GX; ++g) {
          const int xk = (ps.k + 8 * g) * V;
          // every window of the row goes to shared memory (read or not)
          for (int i = 0; i < V; ++i) {
            const int64_t si = static_cast<int64_t>(y + PD) * T.LD + xk - sh + i + PD;
            if (si < 0 || si >= smem_elems) return 318;
            if (si / T.LD != y + PD) return 331;   // stays inside its own row
          }
          if (!(xk - sh < limX)) continue;           // not read
          const int64_t w = row - sh + xk;
          if (md(misA + w) != 0) return 316;        // 16-byte aligned window
          if (!window_ok(w, L.nA)) return 317;     // inside the buffer's blocks
          for (int i = 0; i < V; ++i) {
            const int x = xk - sh + i;
            const int64_t si = static_cast<int64_t>(y + PD) * T.LD + x + PD;
            if (x < 0 || x >= limX) continue;      // padding, never read
            if (slot[si] >= 0) return 319;         // two writers of one slot
            const int64_t ia = w + i;
            if (ia < 0 || ia >= L.nA) return 320;
            if (ia != row + x) return 321;
            slot[si] = ia;
          }
        }
      }
    }
    for (int t = 0; t < T.nt; ++t) {
      const VtPos ps = vt_pos(t);
      if (ps.k >= 8 || ps.r0 >= T.R2) return 322;
      for (int j = 0; j < T.J2; ++j) {
        const int x = ps.r0 + j * T.R2;
        if (!(x < limX)) continue;
        const int64_t col = o.bB + static_cast<int64_t>(tabX[x]);  // element index in B
        const int tt = md(misB + col);
        for (int g = 0; g < GY; ++g) {
        const int yk = (ps.k + 8 * g) * V;
        const int y0 = yk - tt;
        if (!(y0 < limY)) continue;
        const int64_t w = col - tt + yk;
        if (md(misB + w) != 0) return 323;
        if (update && !window_ok(w, L.nB)) return 324;  // the B window read
        const bool full = y0 >= 0 && y0 + V <= limY;
        for (int i = 0; i < V; ++i) {
          const int y = y0 + i;
          const int64_t si = static_cast<int64_t>(y + PD) * T.LD + x + PD;
          if (si < 0 || si >= smem_elems) return 325;
          if (y < 0 || y >= limY) continue;      // not stored
          const int64_t ia = slot[si];
          if (ia < 0) return 326;                // reads a slot no load wrote
          const int64_t ib = w + i;
          if (ib < 0 || ib >= L.nB) return 327;
          if (ib != col + y) return 328;
          if (map_a_to_b(L, ia) != ib) return 329;
          if (writes[ib] != 0) return 330;
          writes[ib] = 1;
          ++*checked;
        }
        (void)full;
        }
      }
    }
  }
  return 0;
}

// TMA tile (ttile.cuh): both tensor maps as the launcher encodes them
// (ttile_map_params), checked against the rules TMA imposes -- unit element
// stride innermost, other strides multiples of 16 bytes, 128-byte inner box
// rows, innermost coordinates of every load and store multiples of 16
// bytes, no negative coordinate -- then every box of every tile, clipped at
// the tensor's edges as TMA clips it, with A and B addresses computed from
// the maps: every inner element of B written exactly once, with the element
// of A the permutation maps to it.  (The persistent form walks tiles
// blockIdx.x + i * gridDim.x, each tile once for any grid, so the same
// per-tile check covers it.)
int replay_ttile(const HpttProblem &P, const HpttTile &T, const Layout &L, int update,
                 std::vector<uint8_t> &writes, uint64_t *checked) {
  const int esz = elem_bytes(P.dtype);
  const int BOX = 128 / esz;
  TtileMapParams ma, mb;
  if (ttile_map_params(P, T, 0, &ma) != ST_OK || ttile_map_params(P, T, 1, &mb) != ST_OK)
    return 401;
  if (ma.rank != P.rank || mb.rank != P.rank || ma.rank > 5) return 402;
  if (ma.stride_bytes[0] != static_cast<uint64_t>(esz) ||
      mb.stride_bytes[0] != static_cast<uint64_t>(esz))
    return 403;
  uint64_t boxa = 1, boxb = 1;
  for (int k = 0; k < P.rank; ++k) {
    if (k > 0 && (ma.stride_bytes[k] % 16 || mb.stride_bytes[k] % 16)) return 404;
    boxa *= ma.box[k];
    boxb *= mb.box[k];
  }
  if (ma.box[0] * esz != 128 || mb.box[0] * esz != 128) return 405;
  if (boxa != static_cast<uint64_t>(BOX) * BOX || boxb != boxa) return 406;
  const int K = T.tkx * T.tky;
  if (K < 1 || K > 8 || (!T.ts && T.nt != 64 * K)) return 407;
  // shared memory: one CTA per tile, two boxes per box of the tile; the
  // persistent form, ts stages (A's boxes, and B's when B is read) and three
  // output buffers; both with the header and alignment slack
  const int kb = K * BOX * 128;
  const int64_t need = T.ts ? int64_t(T.ts) * kb * (update ? 2 : 1) + 3 * kb + 1024 + 256
                            : 2 * kb + 1024 + 16;
  if (T.ts < 0 || T.ts == 1 || T.ts > 4 || T.smem_bytes < need) return 408;
  if (T.ts && (K > 4 || T.nt != 64 * K + 32)) return 415;
  const int p0 = P.perm[0];
  for (uint32_t tile = 0; tile < T.num_tiles; ++tile) {
    int32_t org[5];
    ttile_coords(T, tile, org);
    for (int g = 0; g < K; ++g) {
      int32_t ca[5], cb[5];
      for (int d = 0; d < 5; ++d) ca[d] = org[d];
      ca[0] += (g % T.tkx) * BOX;
      ca[p0] += (g / T.tkx) * BOX;
      if (!(ca[0] < P.n[0] && ca[p0] < P.n[p0])) continue;  // the kernel skips it
      for (int k = 0; k < P.rank; ++k) cb[k] = ca[P.perm[k]];
      for (int k = 0; k < P.rank; ++k)
        if (ca[k] < 0 || cb[k] < 0) return 409;
      if ((static_cast<int64_t>(ca[0]) * esz) % 16 || (static_cast<int64_t>(cb[0]) * esz) % 16)
        return 410;
      for (int y = 0; y < BOX; ++y) {
        for (int x = 0; x < BOX; ++x) {
          int64_t c[5];
          for (int d = 0; d < P.rank; ++d) c[d] = ca[d];
          c[0] += x;
          c[p0] += y;
          if (c[0] >= P.n[0] || c[p0] >= P.n[p0]) continue;  // clipped by TMA
          uint64_t oa = 0, ob = 0;
          for (int k = 0; k < P.rank; ++k) {
            oa += static_cast<uint64_t>(c[k]) * ma.stride_bytes[k];
            ob += static_cast<uint64_t>(c[P.perm[k]]) * mb.stride_bytes[k];
          }
          const int64_t ia = static_cast<int64_t>(oa / esz), ib = static_cast<int64_t>(ob / esz);
          if (ia < 0 || ia >= L.nA) return 411;
          if (ib < 0 || ib >= L.nB) return 412;
          if (map_a_to_b(L, ia) != ib) return 413;
          if (writes[ib] != 0) return 414;
          writes[ib] = 1;
          ++*checked;
        }
      }
    }
  }
  return 0;
}

template <typename OffT>
int replay_rows(const HpttProblem &P, const HpttTile &T, const Layout &L,
                const std::vector<unsigned char> &tab, std::vector<uint8_t> &writes,
                uint64_t *checked) {
  const int vec = T.vec;
  const int esz = elem_bytes(P.dtype);
  const int J = hptt_jmax_rows(esz * vec);
  if (T.J1 > J) return 201;
  if (T.tab2_off < T.TY * static_cast<int>(sizeof(OffT))) return 202;
  if (T.table_bytes < T.tab2_off + T.TY * static_cast<int>(sizeof(OffT))) return 203;
  if (vec > 1 && (P.sA[0] != 1 || P.sB[0] != 1)) return 204;
  const OffT *tabA = reinterpret_cast<const OffT *>(tab.data());
  const OffT *tabB = reinterpret_cast<const OffT *>(tab.data() + T.tab2_off);
  for (uint32_t tile = 0; tile < T.num_tiles; ++tile) {
    const TileOrigin o = tile_origin(P, T, tile);
    const int limY = rows_limit_y(T, o);
    for (int t = 0; t < T.nt; ++t) {
      const RowThread s = rows_thread(T, t);
      if (!s.active) continue;
      const int64_t col = static_cast<int64_t>(s.e) * vec;
      if (col >= o.remX) continue;
      const int n = std::min(T.J1, valid_iters(limY, s.y0, T.r1_mul, T.r1_shr, T.R1));
      // interior tiles run J1 iterations and test only the last one
      if (limY == T.TY && n < T.J1 - 1) return 213;
      for (int j = 0; j < J; ++j) {
        const int y = s.y0 + j * T.R1;
        if (!(j < n)) continue;
        if (!(j < T.J1 && y < limY)) return 212;
        if (y < 0 || y >= T.TY) return 205;
        const int64_t a0 = o.bA + col * P.sA[0] + static_cast<int64_t>(tabA[y]);
        const int64_t b0 = o.bB + col * P.sB[0] + static_cast<int64_t>(tabB[y]);
        if (vec > 1 && ((a0 % vec) != 0 || (b0 % vec) != 0)) return 206;
        for (int k = 0; k < vec; ++k) {
          const int64_t ia = a0 + k, ib = b0 + k;
          if (ia < 0 || ia >= L.nA) return 207;
          if (ib < 0 || ib >= L.nB) return 208;
          if (map_a_to_b(L, ia) != ib) return 209;
          if (writes[ib] != 0) return 210;
          writes[ib] = 1;
          ++*checked;
        }
      }
    }
  }
  return 0;
}

}  // namespace
}  // namespace hptt_b200

using namespace hptt_b200;

namespace hptt_b200 {
namespace {

// Guard, fusion and the host-side layout of a replayed problem.
int replay_setup(int dtype, uint32_t rank, const uint32_t *in_size, const uint32_t *perm,
                 const uint32_t *in_outer, const uint32_t *out_outer, HpttProblem *P,
                 Layout *Lp, std::vector<uint8_t> *inner) {
  if (elem_bytes(dtype) == 0) return HPTT_ERR_DTYPE;
  int st = validate(static_cast<int>(rank), in_size, perm, in_outer, out_outer,
                    in_outer ? static_cast<int>(rank) : 0, out_outer ? static_cast<int>(rank) : 0);
  if (st != ST_OK) return st;
  st = fuse(dtype, static_cast<int>(rank), in_size, perm, in_outer, out_outer, P);
  if (st != ST_OK) return st;
  Layout &L = *Lp;
  L.rank = static_cast<int>(rank);
  for (uint32_t d = 0; d < rank; ++d) {
    L.in_size.push_back(in_size[d]);
    L.in_outer.push_back(in_outer ? in_outer[d] : in_size[d]);
    L.perm.push_back(perm[d]);
  }
  for (uint32_t k = 0; k < rank; ++k)
    L.out_outer.push_back(out_outer ? out_outer[k] : in_size[perm[k]]);
  for (uint32_t d = 0; d < rank; ++d) L.nA *= L.in_outer[d];
  int64_t s = 1;
  for (uint32_t k = 0; k < rank; ++k) {
    L.sbo.push_back(s);
    s *= L.out_outer[k];
  }
  L.nB = s;
  // which B elements are inside the tensor (not outer-size padding)
  inner->assign(static_cast<size_t>(L.nB), 0);
  for (int64_t ib = 0; ib < L.nB; ++ib) (*inner)[ib] = b_is_inner(L, ib) ? 1 : 0;
  return ST_OK;
}

// Replays one vector tile with the given base misalignments; 0 or a code.
int replay_vtile_form(const HpttProblem &P, const Layout &L, const std::vector<uint8_t> &inner,
                      const HpttTile &T, int update, int misA, int misB, uint64_t *checked) {
  std::vector<unsigned char> tab;
  build_tables(P, T, &tab);
  std::vector<uint8_t> writes(static_cast<size_t>(L.nB), 0);
  uint64_t n = 0;
  const int rc = T.big_offsets
                     ? replay_vtile<int64_t>(P, T, update, L, tab, writes, &n, misA, misB)
                     : replay_vtile<uint32_t>(P, T, update, L, tab, writes, &n, misA, misB);
  if (rc != 0) return 2000 + rc;
  for (int64_t ib = 0; ib < L.nB; ++ib)
    if (writes[ib] != inner[ib]) return 2300;
  if (checked) *checked = n;
  return 0;
}

}  // namespace
}  // namespace hptt_b200

extern "C" int hptt_cuda_debug_check_indexing(int dtype, uint32_t rank, const uint32_t *in_size,
                                              const uint32_t *perm, const uint32_t *in_outer,
                                              const uint32_t *out_outer, int max_vec_bytes,
                                              uint64_t *checked) {
  HpttProblem P;
  Layout L;
  std::vector<uint8_t> inner;
  int st = replay_setup(dtype, rank, in_size, perm, in_outer, out_outer, &P, &L, &inner);
  if (st != ST_OK) return st;
  TileParams tp;
  if (max_vec_bytes > 0) tp.max_vec_bytes = max_vec_bytes;
  // every planner knob the tuner tries: side order, both update settings,
  // both per-thread iteration limits, the whole-extent options, tables or
  // walks for two-dim sides, exact or predicated update interiors, 256 or
  // 512 threads per CTA, grid levels in input or stride order
  for (int v = 0; v < 48; ++v) {
    const int variant = v % 24;
    tp.nt = v < 24 ? 256 : 512;
    tp.grid_order = v < 24 ? 0 : 1;
    // 512 threads: the default iteration limit only
    if (v >= 24 && ((variant >> 2) & 1)) continue;
    const int update = variant & 1;
    tp.y_first = (variant >> 1) & 1;
    tp.max_iters = ((variant >> 2) & 1) ? hptt_jmax_tile(elem_bytes(P.dtype)) / 2 : 0;
    tp.full_side = variant >> 3;
    // the tuner's alternative forms, each in half of the variants
    tp.walk = ((variant >> 2) & 1) ? 0 : 1;
    tp.upd_exact = ((variant >> 1) & 1) ? 0 : 1;
    HpttTile T;
    st = choose_tile(P, tp, update, &T);
    if (st != ST_OK) return st;
    std::vector<unsigned char> tab;
    build_tables(P, T, &tab);
    // the single-transpose kernel, then (tiles) the batch kernels' forms
    // (512-thread tiles are planned again for 256 threads in a batch)
    for (int model = 0; model < (T.kind == KIND_TILE && T.nt == 256 ? 2 : 1); ++model) {
      std::vector<uint8_t> writes(static_cast<size_t>(L.nB), 0);
      uint64_t n = 0;
      int rc;
      const bool fast = model == 0;
      if (T.kind == KIND_TILE)
        rc = T.big_offsets ? replay_tile<int64_t>(P, T, update, L, tab, writes, &n, fast)
                           : replay_tile<uint32_t>(P, T, update, L, tab, writes, &n, fast);
      else
        rc = T.big_offsets ? replay_rows<int64_t>(P, T, L, tab, writes, &n)
                           : replay_rows<uint32_t>(P, T, L, tab, writes, &n);
      if (rc != 0) return 1000 + rc + (model ? 500 : 0);
      for (int64_t ib = 0; ib < L.nB; ++ib)
        if (writes[ib] != inner[ib]) return 1300;
      if (checked) *checked = n;
    }
  }
  // vector tiles: window-slot shapes and thread counts the tuner tries, both
  // grid orders, and A/B base addresses on and off a 16-byte boundary.  The
  // vector tile's shape does not depend on whether B is read, so one replay
  // with the B-window checks covers both settings.
  if (vtile_possible(P)) {
    const int V = 16 / elem_bytes(P.dtype);
    const int shapes[][5] = {{256, 16, 16, 0, 8}, {256, 16, 32, 1, 4}, {512, 32, 32, 0, 8},
                             {256, 32, 8, 1, 8},  {512, 8, 32, 0, 4}};
    for (const auto &sh : shapes) {
      {
        const int update = 1;
        TileParams vp;
        vp.vt = 1;
        vp.nt = sh[0];
        vp.vt_nvx = sh[1];
        vp.vt_nvy = sh[2];
        vp.grid_order = sh[3];
        vp.vt_j = sh[4];
        HpttTile T;
        st = choose_tile(P, vp, update, &T);
        if (st != ST_OK) return st;
        if (T.kind != KIND_VTILE) continue;  // the tile form, replayed above
        for (int m = 0; m < 4; ++m) {
          const int misA = (m & 1) ? V - 1 : 0;
          const int misB = (m == 1 || m == 2) ? V - 1 : (m == 3 ? 1 : 0);
          uint64_t n = 0;
          const int rc = replay_vtile_form(P, L, inner, T, update, misA, misB, &n);
          if (rc != 0) return rc;
          if (checked && *checked != n) return 2301;
        }
      }
    }
  }
  // TMA tiles: boxes per tile and both grid orders
  if (ttile_possible(P)) {
    // (boxes along input dim 0, along the output's leading dim, grid order,
    // stages, B read)
    const int forms[][5] = {{1, 1, 0, 1, 0}, {2, 2, 1, 1, 1}, {4, 2, 0, 1, 0}, {1, 4, 1, 2, 1},
                            {2, 1, 0, 4, 0}, {1, 1, 0, 3, 1}, {2, 2, 1, 2, 0}};
    for (const auto &f : forms) {
      TileParams tp2;
      tp2.tt = f[3];
      tp2.tt_kx = f[0];
      tp2.tt_ky = f[1];
      tp2.grid_order = f[2];
      HpttTile T;
      st = choose_tile(P, tp2, f[4], &T);
      if (st != ST_OK) return st;
      if (T.kind != KIND_TTILE) return 2400;
      std::vector<uint8_t> writes(static_cast<size_t>(L.nB), 0);
      uint64_t n = 0;
      const int rc = replay_ttile(P, T, L, f[4], writes, &n);
      if (rc != 0) return 2000 + rc;
      for (int64_t ib = 0; ib < L.nB; ++ib)
        if (writes[ib] != inner[ib]) return 2401;
      if (checked && *checked != n) return 2402;
    }
  }
  return 0;
}

extern "C" int hptt_cuda_debug_check_vtile(int dtype, uint32_t rank, const uint32_t *in_size,
                                           const uint32_t *perm, const uint32_t *in_outer,
                                           const uint32_t *out_outer, int nt, int nvx, int nvy,
                                           int vj, int grid_order, int update, int mis_a,
                                           int mis_b, uint64_t *checked) {
  HpttProblem P;
  Layout L;
  std::vector<uint8_t> inner;
  if (checked) *checked = 0;
  int st = replay_setup(dtype, rank, in_size, perm, in_outer, out_outer, &P, &L, &inner);
  if (st != ST_OK) return st;
  TileParams vp;
  vp.vt = 1;
  vp.nt = nt;
  vp.vt_nvx = nvx;
  vp.vt_nvy = nvy;
  vp.vt_j = vj;
  vp.grid_order = grid_order;
  HpttTile T;
  st = choose_tile(P, vp, update, &T);
  if (st != ST_OK) return st;
  if (T.kind != KIND_VTILE) return 0;
  return replay_vtile_form(P, L, inner, T, update, mis_a, mis_b, checked);
}
