// Per-plan offset tables, computed on the host from the planner's index maps
// (tile_maps / tile_thread_consts) and the row helpers in kernels.cuh.
#include "tables.h"

#include <cstring>

#include "kernels.cuh"
#include "planner.h"

namespace hptt_b200 {

namespace {

template <typename OffT>
void build_typed(const HpttProblem &P, const HpttTile &T, unsigned char *base) {
  if (T.kind == KIND_TILE) {
    TileMaps m;
    tile_maps(P, T, &m);
    HpttTabEnt<OffT> *ld = reinterpret_cast<HpttTabEnt<OffT> *>(base);
    HpttTabEnt<OffT> *st = reinterpret_cast<HpttTabEnt<OffT> *>(base + T.tab2_off);
    for (int q = 0; q < T.TY; ++q) {
      ld[q].off = static_cast<OffT>(m.offA[q]);
      ld[q].c = m.cy[q];
    }
    for (int q = 0; q < T.TX; ++q) {
      st[q].off = static_cast<OffT>(m.offB[q]);
      st[q].c = m.cx[q];
    }
    HpttThr *thr = reinterpret_cast<HpttThr *>(base + T.thr_off);
    for (int t = 0; t < T.nt; ++t) thr[t] = tile_thread_consts(P, T, m, t);
  } else if (T.kind == KIND_TTILE) {
    // no tables: TMA addresses both tensors from the tile coordinates
  } else if (T.kind == KIND_VTILE) {
    std::vector<int64_t> rowA, colB;
    vtile_maps(P, T, &rowA, &colB);
    OffT *ra = reinterpret_cast<OffT *>(base);
    OffT *cb = reinterpret_cast<OffT *>(base + T.tab2_off);
    for (int y = 0; y < T.TY; ++y) ra[y] = static_cast<OffT>(rowA[y]);
    for (int x = 0; x < T.TX; ++x) cb[x] = static_cast<OffT>(colB[x]);
  } else {
    dev::rows_tables<OffT>(P, T, reinterpret_cast<OffT *>(base),
                           reinterpret_cast<OffT *>(base + T.tab2_off), 0, 1);
  }
}

}  // namespace

void build_tables(const HpttProblem &P, const HpttTile &T, std::vector<unsigned char> *out) {
  out->assign(static_cast<size_t>(T.table_bytes), 0);
  if (T.big_offsets)
    build_typed<int64_t>(P, T, out->data());
  else
    build_typed<uint32_t>(P, T, out->data());
}

}  // namespace hptt_b200
