// Host planner: argument guard, index fusion, tile and grid selection.
//
// This replaces the reference's CPU planning layer
//   - argument guard            src/hptt.cc:25-56
//   - index fusion              inc/hptt/param/parameter_trans.tcc:223-283, 65-97
//   - loop-order / thread split inc/hptt/plan/plan_trans_util.tcc (whole file)
// with a GPU tile and grid chooser.  The fusion rule is the reference's
// (adjacent-and-in-order under perm, unpadded) stated on strides: two
// neighbouring output dims fuse when they are consecutive input dims and the
// upper one's stride equals the lower one's stride times its extent in both
// A and B.  Extent-1 dims are dropped first (they never change an offset).
#include "planner.h"
#include "vtile.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <vector>

namespace hptt_b200 {


const char *status_string(int st) {
  switch (st) {
    case ST_OK: return "ok";
    case ST_NULL_DATA: return "null data pointer";
    case ST_BAD_RANK: return "tensor rank must be >= 2 (and <= 8)";
    case ST_BAD_SIZE_VECTOR: return "size vector length does not match the rank";
    case ST_BAD_SIZE_VALUE: return "zero extent or outer size below inner size";
    case ST_BAD_PERM: return "perm is not a permutation of 0..rank-1";
    case ST_BAD_DTYPE: return "unknown element type";
    case ST_CUDA: return "CUDA runtime error";
    case ST_NO_DEVICE: return "no CUDA device";
    case ST_ALLOC: return "allocation failed";
    case ST_BUDGET: return "request exceeds the memory budget";
    case ST_BAD_HANDLE: return "invalid handle";
    case ST_TIMEOUT: return "bounded wait ran out";
    case ST_TOO_LARGE: return "size beyond what this build supports";
    case ST_BUSY: return "no free slot";
    case ST_LABELS: return "contraction labels do not describe a contraction";
    case ST_BLAS: return "cuBLAS call failed";
    default: return "unknown status";
  }
}

int elem_bytes(int dtype) {
  switch (dtype) {
    case DT_F32: return 4;
    case DT_F64: return 8;
    case DT_C64: return 8;
    case DT_C128: return 16;
    default: return 0;
  }
}

int validate(int rank, const uint32_t *in_size, const uint32_t *perm,
             const uint32_t *in_outer, const uint32_t *out_outer,
             int in_outer_len, int out_outer_len) {
  // Order checks follow src/hptt.cc:30-56.  The permutation is validated
  // before it is used as an index (the reference reads out_outer[perm[i]]
  // first); both orders reject the same inputs.
  if (rank <= 1) return ST_BAD_RANK;
  if (rank > HPTT_MAX_RANK) return ST_BAD_RANK;
  if (!in_size || !perm) return ST_BAD_SIZE_VECTOR;
  if ((in_outer_len != 0 && in_outer_len != rank) ||
      (out_outer_len != 0 && out_outer_len != rank))
    return ST_BAD_SIZE_VECTOR;
  if ((in_outer_len != 0 && !in_outer) || (out_outer_len != 0 && !out_outer))
    return ST_BAD_SIZE_VECTOR;
  bool seen[HPTT_MAX_RANK] = {false};
  bool perm_ok = true;
  for (int k = 0; k < rank; ++k) {
    if (perm[k] >= static_cast<uint32_t>(rank) || seen[perm[k]]) {
      perm_ok = false;
      break;
    }
    seen[perm[k]] = true;
  }
  if (perm_ok) {
    for (int i = 0; i < rank; ++i) {
      if (in_size[i] == 0) return ST_BAD_SIZE_VALUE;
      if (in_outer_len && in_outer[i] < in_size[i]) return ST_BAD_SIZE_VALUE;
      // reference check, src/hptt.cc:47-49
      if (out_outer_len && out_outer[perm[i]] < in_size[i]) return ST_BAD_SIZE_VALUE;
    }
    // memory-safety check the reference omits: output dim k has extent
    // in_size[perm[k]] (hptt_trans_gen.py:196-197).
    if (out_outer_len)
      for (int k = 0; k < rank; ++k)
        if (out_outer[k] < in_size[perm[k]]) return ST_BAD_SIZE_VALUE;
    return ST_OK;
  }
  for (int i = 0; i < rank; ++i)
    if (in_size[i] == 0) return ST_BAD_SIZE_VALUE;
  return ST_BAD_PERM;
}

int fuse(int dtype, int rank, const uint32_t *in_size, const uint32_t *perm,
         const uint32_t *in_outer, const uint32_t *out_outer,
         HpttProblem *out) {
  if (elem_bytes(dtype) == 0) return ST_BAD_DTYPE;
  int64_t n[HPTT_MAX_RANK], sA[HPTT_MAX_RANK], sB[HPTT_MAX_RANK];
  int q[HPTT_MAX_RANK];
  int64_t s = 1;
  for (int d = 0; d < rank; ++d) {
    n[d] = in_size[d];
    sA[d] = s;
    s *= in_outer ? in_outer[d] : in_size[d];
  }
  s = 1;
  int64_t sBout[HPTT_MAX_RANK];
  for (int k = 0; k < rank; ++k) {
    q[perm[k]] = k;
    sBout[k] = s;
    s *= out_outer ? out_outer[k] : in_size[perm[k]];
  }
  for (int d = 0; d < rank; ++d) sB[d] = sBout[q[d]];

  // Input dims in output order, extent-1 dims dropped.
  std::vector<int> ord;
  for (int k = 0; k < rank; ++k)
    if (n[perm[k]] > 1) ord.push_back(static_cast<int>(perm[k]));

  std::memset(out, 0, sizeof(*out));
  out->dtype = dtype;
  if (ord.empty()) {  // a single element
    out->rank = 1;
    out->n[0] = 1;
    out->sA[0] = 1;
    out->sB[0] = 1;
    out->perm[0] = 0;
    return ST_OK;
  }
  // next kept input dim after d (input order)
  auto next_kept = [&](int d) {
    for (int e = d + 1; e < rank; ++e)
      if (n[e] > 1) return e;
    return -1;
  };
  struct Group { int first, last; int64_t ext; };
  std::vector<Group> groups;  // in output order
  for (int d : ord) {
    if (!groups.empty()) {
      Group &g = groups.back();
      const int prev = g.last;
      if (next_kept(prev) == d && sA[d] == sA[prev] * n[prev] &&
          sB[d] == sB[prev] * n[prev]) {
        g.last = d;
        g.ext *= n[d];
        continue;
      }
    }
    groups.push_back({d, d, n[d]});
  }
  // groups sorted by first input dim -> fused input dims
  std::vector<int> by_in(groups.size());
  for (size_t i = 0; i < groups.size(); ++i) by_in[i] = static_cast<int>(i);
  std::sort(by_in.begin(), by_in.end(), [&](int a, int b) {
    return groups[a].first < groups[b].first;
  });
  std::vector<int> id_of_group(groups.size());
  out->rank = static_cast<int32_t>(groups.size());
  for (size_t i = 0; i < by_in.size(); ++i) {
    const Group &g = groups[by_in[i]];
    id_of_group[by_in[i]] = static_cast<int>(i);
    out->n[i] = g.ext;
    out->sA[i] = sA[g.first];
    out->sB[i] = sB[g.first];
  }
  for (size_t k = 0; k < groups.size(); ++k) out->perm[k] = id_of_group[k];
  return ST_OK;
}

namespace {

// Enumerate the digits of a tile-local mixed-radix index in a chosen order.
//   dims/ext: the side's dims and tile extents in the side's own order (the
//   index's radix order, first fastest); order: permutation of 0..nd-1 giving
//   the enumeration order (first fastest).  For every slot q, returns the
//   index in the side's own order, its offset with `stride`, and its
//   coordinate along `chunk_dim` (0 when that dim is not on this side).
void enumerate(int nd, const int32_t *dims, const int32_t *ext, const int *order,
               const int64_t *stride, int chunk_dim, std::vector<int> *idx,
               std::vector<int64_t> *off, std::vector<int> *chunk) {
  int64_t place[HPTT_MAX_RANK];
  int64_t total = 1;
  for (int i = 0; i < nd; ++i) {
    place[i] = total;
    total *= ext[i];
  }
  idx->assign(static_cast<size_t>(total), 0);
  off->assign(static_cast<size_t>(total), 0);
  chunk->assign(static_cast<size_t>(total), 0);
  for (int64_t q = 0; q < total; ++q) {
    int64_t rem = q, id = 0, o = 0;
    int cc = 0;
    for (int k = 0; k < nd; ++k) {
      const int i = order[k];
      const int64_t c = rem % ext[i];
      rem /= ext[i];
      id += c * place[i];
      o += c * stride[dims[i]];
      if (dims[i] == chunk_dim) cc = static_cast<int>(c);
    }
    (*idx)[q] = static_cast<int>(id);
    (*off)[q] = o;
    (*chunk)[q] = cc;
  }
}

// Coordinate of side-order index `idx` along `chunk_dim`, and its offset.
int64_t side_offset(int idx, int nd, const int32_t *dims, const int32_t *ext,
                    const int64_t *stride, int chunk_dim, int *chunk) {
  int64_t o = 0;
  *chunk = 0;
  for (int i = 0; i < nd; ++i) {
    const int c = idx % ext[i];
    idx /= ext[i];
    o += static_cast<int64_t>(c) * stride[dims[i]];
    if (dims[i] == chunk_dim) *chunk = c;
  }
  return o;
}

}  // namespace

void tile_maps(const HpttProblem &p, const HpttTile &t, TileMaps *m) {
  int order[HPTT_MAX_RANK];
  std::vector<int> slot_to_y, slot_to_x;
  // rows: Y dims in input order
  for (int i = 0; i < t.ny; ++i) order[i] = i;
  std::sort(order, order + t.ny, [&](int a, int b) { return t.yd[a] < t.yd[b]; });
  enumerate(t.ny, t.yd, t.yt, order, p.sA, t.yc, &slot_to_y, &m->offA, &m->cy);
  // columns: X dims in output order
  int pos[HPTT_MAX_RANK];
  for (int k = 0; k < p.rank; ++k) pos[p.perm[k]] = k;
  for (int i = 0; i < t.nx; ++i) order[i] = i;
  std::sort(order, order + t.nx, [&](int a, int b) { return pos[t.xd[a]] < pos[t.xd[b]]; });
  enumerate(t.nx, t.xd, t.xt, order, p.sB, t.xc, &slot_to_x, &m->offB, &m->cx);
  m->qrow.assign(slot_to_y.size(), 0);
  for (size_t q = 0; q < slot_to_y.size(); ++q) m->qrow[slot_to_y[q]] = static_cast<int>(q);
  m->qcol.assign(slot_to_x.size(), 0);
  for (size_t q = 0; q < slot_to_x.size(); ++q) m->qcol[slot_to_x[q]] = static_cast<int>(q);
}

HpttThr tile_thread_consts(const HpttProblem &p, const HpttTile &t, const TileMaps &m,
                           int tid) {
  HpttThr h;
  std::memset(&h, 0, sizeof(h));
  const bool ld = tid < t.R1 * t.RW, st = tid < t.R2 * t.WTY;
  h.active = (ld ? 1 : 0) | (st ? 2 : 0);
  {
    const int e = tid % t.RW, w = e % t.W, x = e / t.W;
    h.q0 = tid / t.RW;
    h.inE = side_offset(x, t.nx, t.xd, t.xt, p.sA, t.xc, &h.cxe) +
            static_cast<int64_t>(w) * p.sA[0];
    h.sme = m.qcol[x] * t.W + w;
  }
  {
    const int e2 = tid % t.WTY, w = e2 % t.W, y = e2 / t.W;
    h.qs0 = tid / t.WTY;
    h.outE2 = side_offset(y, t.ny, t.yd, t.yt, p.sB, t.yc, &h.cye2) +
              static_cast<int64_t>(w) * p.sB[0];
    h.sme2 = m.qrow[y] * t.LD + w;
  }
  return h;
}

namespace {

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Shared-memory wavefronts for one warp whose lanes access byte addresses
// addr[lane] (each lane `bytes` wide); returns wavefronts beyond the ideal.
int excess_wavefronts(const int64_t *addr, int lanes, int bytes) {
  // count distinct 4-byte words per bank
  std::vector<int64_t> words[32];
  for (int l = 0; l < lanes; ++l) {
    if (addr[l] < 0) continue;
    for (int b = 0; b < bytes; b += 4) {
      const int64_t w = (addr[l] + b) / 4;
      auto &v = words[w % 32];
      if (std::find(v.begin(), v.end(), w) == v.end()) v.push_back(w);
    }
  }
  size_t worst = 0;
  int active = 0;
  for (int l = 0; l < lanes; ++l) active += addr[l] >= 0;
  for (auto &v : words) worst = std::max(worst, v.size());
  const int ideal = static_cast<int>(cdiv(static_cast<int64_t>(active) * bytes, 128));
  return static_cast<int>(worst) - std::max(ideal, 1);
}

// Shared-memory wavefronts beyond the ideal for the first warps of both
// phases with row pitch `ld` (same addressing as tile_one).
int bank_cost(const HpttTile &t, int ld, int sz, const TileMaps &m) {
  int cost = 0;
  int64_t addr[32];
  const int warps = std::min(t.nt / 32, 4);
  for (int w = 0; w < warps; ++w) {
    // load phase: thread (e, q0) writes row slot q0 at column qcol(x)*W + w
    for (int l = 0; l < 32; ++l) {
      const int tid = w * 32 + l;
      if (tid < t.R1 * t.RW) {
        const int e = tid % t.RW, q = tid / t.RW;
        const int col = m.qcol[e / t.W] * t.W + e % t.W;
        addr[l] = (q < t.TY) ? static_cast<int64_t>(q * ld + col) * sz : -1;
      } else {
        addr[l] = -1;
      }
    }
    cost += excess_wavefronts(addr, 32, sz);
    // store phase: thread (e2, qs0) reads row qrow(y) at column qs0*W + w
    for (int l = 0; l < 32; ++l) {
      const int tid = w * 32 + l;
      if (tid < t.R2 * t.WTY) {
        const int e2 = tid % t.WTY, q = tid / t.WTY;
        const int ww = e2 % t.W, y = e2 / t.W;
        addr[l] = (q < t.TX) ? static_cast<int64_t>(m.qrow[y] * ld + ww + t.W * q) * sz : -1;
      } else {
        addr[l] = -1;
      }
    }
    cost += excess_wavefronts(addr, 32, sz);
  }
  return cost;
}

struct Side {
  std::vector<int> d;
  std::vector<int64_t> t;
  int64_t prod() const {
    int64_t p = 1;
    for (auto v : t) p *= v;
    return p;
  }
};

bool shape_ok(const TileParams &tp, int64_t W, const Side &X, const Side &Y,
              int sz) {
  const int kJMax = tp.max_iters > 0 ? std::min(tp.max_iters, hptt_jmax_tile(sz))
                                     : hptt_jmax_tile(sz);
  const int64_t TX = X.prod(), TY = Y.prod();
  const int64_t RW = W * TX, WTY = W * TY;
  if (RW > tp.nt || WTY > tp.nt) return false;
  const int64_t R1 = tp.nt / RW, R2 = tp.nt / WTY;
  if (cdiv(TY, R1) > kJMax || cdiv(TX, R2) > kJMax) return false;
  if (RW * TY * sz > tp.smem_bytes) return false;
  return true;
}

// Division by a run-time constant d as multiply-high and shift, exact for
// dividends below 2^31: with l = ceil(log2 d) and p = 31 + l,
// m = ceil(2^p / d) and n / d = (n * m) >> p.  mul = 0 encodes d == 1.
void fast_div_magic(uint32_t d, uint32_t *mul, int32_t *shr) {
  if (d <= 1) {
    *mul = 0;
    *shr = 0;
    return;
  }
  int l = 0;
  while ((1ull << l) < d) ++l;
  const int pw = 31 + l;
  *mul = static_cast<uint32_t>(((1ull << pw) + d - 1) / d);
  *shr = pw - 32;
}

void finish_grid(const HpttProblem &p, HpttTile *t, const int64_t *tile_ext,
                 const std::vector<int> &chunk_first, int order = 0) {
  // grid dims: chunked tile dims first, then every dim not fully inside the
  // tile in input order (order 0) or by min(|stride in A|, |stride in B|)
  // (order 1: the neighbours that continue a tile's runs in A or in B come
  // next in tile order)
  t->ng = 0;
  bool used[HPTT_MAX_RANK] = {false};
  uint64_t tiles = 1;
  auto add = [&](int d) {
    const int64_t cnt = cdiv(p.n[d], tile_ext[d]);
    used[d] = true;
    if (cnt <= 1) return;
    t->gd[t->ng] = d;
    t->gcnt[t->ng] = static_cast<uint32_t>(cnt);
    t->gstep[t->ng] = static_cast<int32_t>(tile_ext[d]);
    ++t->ng;
    tiles *= static_cast<uint64_t>(cnt);
  };
  for (int d : chunk_first)
    if (d >= 0 && !used[d]) add(d);
  std::vector<int> rest;
  for (int d = 0; d < p.rank; ++d)
    if (!used[d]) rest.push_back(d);
  if (order == 1) {
    auto key = [&](int d) {
      const int64_t a = p.sA[d] < 0 ? -p.sA[d] : p.sA[d];
      const int64_t b = p.sB[d] < 0 ? -p.sB[d] : p.sB[d];
      return std::min(a, b);
    };
    std::stable_sort(rest.begin(), rest.end(), [&](int x, int y) { return key(x) < key(y); });
  }
  for (int d : rest) add(d);
  t->num_tiles = tiles > 0x7fffffffULL ? 0 : static_cast<uint32_t>(tiles);
  for (int g = 0; g < t->ng; ++g) fast_div_magic(t->gcnt[g], &t->gmul[g], &t->gshr[g]);
}

// The fast divisions by R1/R2.  (Tile origins are decoded on the device: a
// per-tile origin table was measured slower -- every CTA's first loads then
// wait on a cold read of its own entry.)
void finish_tables(const HpttProblem &p, HpttTile *t) {
  // grid levels folded for static-offset reads on the device
  const int xc = t->kind == KIND_ROWS ? t->wc : t->xc;
  for (int g = 0; g < HPTT_MAX_RANK; ++g) {
    if (g < t->ng) {
      const int d = t->gd[g];
      t->gsa[g] = static_cast<int64_t>(t->gstep[g]) * p.sA[d];
      t->gsb[g] = static_cast<int64_t>(t->gstep[g]) * p.sB[d];
      t->gn[g] = p.n[d];
      t->gflag[g] = (d == xc ? 1 : 0) | (d == t->yc ? 2 : 0);
    } else {
      t->gsa[g] = t->gsb[g] = 0;
      t->gn[g] = t->gflag[g] = 0;
    }
  }
  t->xce = 1;
  t->yce = 1;
  for (int i = 0; i < t->nx; ++i)
    if (t->xd[i] == t->xc) t->xce = t->xt[i];
  for (int i = 0; i < t->ny; ++i)
    if (t->yd[i] == t->yc) t->yce = t->yt[i];
  t->sxa = t->nx == 1 ? p.sA[t->xd[0]] : 0;
  t->sxb = t->nx == 1 ? p.sB[t->xd[0]] : 0;
  t->sya = t->ny == 1 ? p.sA[t->yd[0]] : 0;
  t->syb = t->ny == 1 ? p.sB[t->yd[0]] : 0;
  fast_div_magic(static_cast<uint32_t>(t->R1 > 0 ? t->R1 : 1), &t->r1_mul, &t->r1_shr);
  fast_div_magic(static_cast<uint32_t>(t->R2 > 0 ? t->R2 : 1), &t->r2_mul, &t->r2_shr);
  fast_div_magic(static_cast<uint32_t>(t->TX > 0 ? t->TX : 1), &t->tx_mul, &t->tx_shr);
  fast_div_magic(static_cast<uint32_t>(t->TY > 0 ? t->TY : 1), &t->ty_mul, &t->ty_shr);
  // two-dim sides of a tile: walk constants (slot order as in tile_maps: Y
  // dims in input order, X dims in output order)
  std::memset(&t->wx, 0, sizeof(t->wx));
  std::memset(&t->wy, 0, sizeof(t->wy));
  if (t->kind != KIND_TILE || t->big_offsets) return;
  auto walk = [](HpttWalk *w, int i0, int i1, const int32_t *dims, const int32_t *ext,
                 const int64_t *stride, int R) {
    const int64_t e0 = ext[i0], s0 = stride[dims[i0]], s1 = stride[dims[i1]];
    if (R <= 0 || e0 <= 1) return;
    const int64_t r0 = R % e0, r1 = R / e0;
    const int64_t step = r0 * s0 + r1 * s1, carry = s1 - e0 * s0;
    const int64_t lim = 0x7fffffffLL;
    if (step > lim || step < -lim || carry > lim || carry < -lim || e0 * s0 > lim ||
        s1 > lim)
      return;
    w->e0 = static_cast<int32_t>(e0);
    w->r0 = static_cast<int32_t>(r0);
    w->step = static_cast<int32_t>(step);
    w->carry = static_cast<int32_t>(carry);
    w->s0 = static_cast<int32_t>(s0);
    w->s1 = static_cast<int32_t>(s1);
    fast_div_magic(static_cast<uint32_t>(e0), &w->mul, &w->shr);
  };
  if (t->ny == 2) {
    const bool in_order = t->yd[0] < t->yd[1];
    walk(&t->wy, in_order ? 0 : 1, in_order ? 1 : 0, t->yd, t->yt, p.sA, t->R1);
  }
  if (t->nx == 2) {
    int pos[HPTT_MAX_RANK];
    for (int k = 0; k < p.rank; ++k) pos[p.perm[k]] = k;
    const bool in_order = pos[t->xd[0]] < pos[t->xd[1]];
    walk(&t->wx, in_order ? 0 : 1, in_order ? 1 : 0, t->xd, t->xt, p.sB, t->R2);
  }
}

int choose_rows(const HpttProblem &p, const TileParams &tp, HpttTile *t) {
  const int sz = elem_bytes(p.dtype);
  std::memset(t, 0, sizeof(*t));
  t->kind = KIND_ROWS;
  t->nt = tp.nt;
  t->xc = t->yc = t->wc = -1;
  const int64_t n0 = p.n[0];
  // widest vector (<= 16 bytes) that divides the row and every other stride
  int vec = std::max(1, std::min(16, tp.max_vec_bytes) / sz);
  while (vec > 1) {
    bool ok = (n0 % vec == 0) && p.sA[0] == 1 && p.sB[0] == 1;
    for (int d = 1; d < p.rank && ok; ++d)
      ok = (p.sA[d] % vec == 0) && (p.sB[d] % vec == 0);
    if (ok) break;
    vec /= 2;
  }
  t->vec = vec;
  const int64_t nvec_row = n0 / vec;
  int64_t wv = std::min<int64_t>(nvec_row, tp.nt);  // vectors per tile row
  t->W = static_cast<int32_t>(wv * vec);
  if (t->W < n0) t->wc = 0;
  t->RW = static_cast<int32_t>(wv);  // threads along a row
  t->R1 = static_cast<int32_t>(tp.nt / wv);
  const int kJMax = hptt_jmax_rows(vec * sz);
  // rows: other dims in output order, full then chunked, up to the volume
  const int64_t rows_target = std::max<int64_t>(
      1, std::min<int64_t>(static_cast<int64_t>(t->R1) * kJMax,
                           cdiv(tp.vmin_bytes, static_cast<int64_t>(t->W) * sz)));
  int64_t TY = 1;
  int64_t tile_ext[HPTT_MAX_RANK];
  for (int d = 0; d < p.rank; ++d) tile_ext[d] = 1;
  tile_ext[0] = t->W;
  for (int k = 1; k < p.rank && TY < rows_target; ++k) {
    const int d = p.perm[k];
    const int64_t tt = std::min<int64_t>(p.n[d], rows_target / TY);
    if (tt <= 1) break;
    t->yd[t->ny] = d;
    t->yt[t->ny] = static_cast<int32_t>(tt);
    ++t->ny;
    tile_ext[d] = tt;
    TY *= tt;
    if (tt < p.n[d]) {
      t->yc = d;
      break;
    }
  }
  t->TY = static_cast<int32_t>(TY);
  t->TX = 1;
  t->px = 1;
  t->py = 1;
  for (int i = 0; i + 1 < t->ny; ++i) t->py *= t->yt[i];
  t->J1 = static_cast<int32_t>(cdiv(TY, t->R1));
  t->WTY = t->W;
  t->LD = 0;
  finish_grid(p, t, tile_ext, {t->wc, t->yc}, tp.grid_order);
  // in-tile offsets
  int64_t maxA = (t->W - 1) * p.sA[0], maxB = (t->W - 1) * p.sB[0];
  for (int i = 0; i < t->ny; ++i) {
    maxA += (t->yt[i] - 1) * p.sA[t->yd[i]];
    maxB += (t->yt[i] - 1) * p.sB[t->yd[i]];
  }
  t->big_offsets = (maxA >= 0x7fffffffLL || maxB >= 0x7fffffffLL);
  const int off = t->big_offsets ? 8 : 4;
  t->smem_bytes = 0;
  t->tab2_off = (t->TY * off + 15) & ~15;
  t->thr_off = t->tab2_off + ((t->TY * off + 15) & ~15);
  t->table_bytes = t->thr_off;
  finish_tables(p, t);
  return t->num_tiles ? ST_OK : ST_TOO_LARGE;
}

// Shared-memory wavefronts beyond the ideal of a vector tile's accesses with
// row pitch `ld`: the first row of every thread of the first warps in the
// load phase (each of its window's V elements) and their first column in the
// store phase, with the rows' and columns' window shifts taken from the
// offsets (a tile origin on a 16-byte boundary).
int vtile_bank_cost(const HpttTile &t, int ld, int sz, const std::vector<int64_t> &rowA,
                    const std::vector<int64_t> &colB) {
  const int V = 16 / sz, P = V - 1;
  auto md = [V](int64_t v) { return static_cast<int>(((v % V) + V) % V); };
  int cost = 0;
  int64_t addr[32];
  const int warps = std::min(t.nt / 32, 8);
  for (int w = 0; w < warps; ++w) {
    for (int i = 0; i < V; ++i) {
      // load phase: the warp's first rows, first slot group
      for (int l = 0; l < 32; ++l) {
        const dev::VtPos ps = dev::vt_pos(w * 32 + l);
        const int y = ps.r0;
        addr[l] = -1;
        if (y >= t.TY) continue;
        const int sh = md(rowA[y]);
        if (ps.k * V - sh >= t.TX) continue;
        addr[l] = (static_cast<int64_t>(y + P) * ld + ps.k * V - sh + i + P) * sz;
      }
      cost += excess_wavefronts(addr, 32, sz);
      // store phase: the warp's first columns, first slot group
      for (int l = 0; l < 32; ++l) {
        const dev::VtPos ps = dev::vt_pos(w * 32 + l);
        const int x = ps.r0;
        addr[l] = -1;
        if (x >= t.TX) continue;
        const int y0 = ps.k * V - md(colB[x]);
        if (y0 >= t.TY) continue;
        addr[l] = (static_cast<int64_t>(y0 + i + P) * ld + x + P) * sz;
      }
      cost += excess_wavefronts(addr, 32, sz);
    }
  }
  return cost;
}

int log2_slots(int n) { return n >= 32 ? 2 : (n >= 16 ? 1 : 0); }

// Vector tile (KIND_VTILE, vtile.cuh).  X: input dims 0, 1, ... whose A
// strides chain (one contiguous run of A), never the output's leading dim;
// Y: output dims 0, 1, ... not in X whose B strides chain (one run of B).
// Each side takes whole dims while its run fits the window slots
// (nvx * V - V + 1 elements: any start shift fits) and the other phase's
// per-thread vectors (nt / 8 lines per pass, each line's slots / 8 vectors
// per line, at most vt_j in all), then a balanced chunk of the next dim.
int choose_vtile(const HpttProblem &p, const TileParams &tp, int update, HpttTile *t) {
  const int sz = elem_bytes(p.dtype);
  if (!vtile_possible(p)) return ST_TOO_LARGE;
  const int V = 16 / sz;
  if (tp.vt_j != 4 && tp.vt_j != 8) return ST_TOO_LARGE;
  const int JV = tp.vt_j;
  const int r = p.rank;
  std::memset(t, 0, sizeof(*t));
  t->kind = KIND_VTILE;
  t->vj = JV;
  t->vpre = (tp.vt_pre && update && JV == 4) ? 1 : 0;
  t->nt = tp.nt;
  t->vec = V;
  t->W = 1;
  t->xc = t->yc = t->wc = -1;
  auto fits = [](int n) { return n == 8 || n == 16 || n == 32; };
  if (!fits(tp.vt_nvx) || !fits(tp.vt_nvy)) return ST_TOO_LARGE;
  if (tp.nt != 256 && tp.nt != 512) return ST_TOO_LARGE;
  // lines (rows in the load phase, columns in the store phase) per pass: a
  // warp covers 4, each thread every eighth window slot of its lines, so a
  // thread holds J lines x (slots / 8) vectors
  const int R = tp.nt / 8;
  bool in_x[HPTT_MAX_RANK] = {false};
  int64_t tile_ext[HPTT_MAX_RANK];
  for (int d = 0; d < r; ++d) tile_ext[d] = 1;
  // X run: bounded by the load window and by the store phase's iterations
  const int64_t txmax =
      std::min<int64_t>(tp.vt_nvx * V - V + 1, static_cast<int64_t>(R) * (JV / (tp.vt_nvy / 8)));
  int64_t TX = 1;
  for (int d = 0; d < r; ++d) {
    if (d == p.perm[0]) break;
    if (d == 0 ? p.sA[0] != 1 : p.sA[d] != p.sA[d - 1] * p.n[d - 1]) break;
    if (TX * p.n[d] <= txmax) {
      t->xd[t->nx] = d;
      t->xt[t->nx++] = static_cast<int32_t>(p.n[d]);
      TX *= p.n[d];
      in_x[d] = true;
      continue;
    }
    const int64_t c = txmax / TX;
    if (c >= 2) {
      const int64_t tt = cdiv(p.n[d], cdiv(p.n[d], c));
      t->xd[t->nx] = d;
      t->xt[t->nx++] = static_cast<int32_t>(tt);
      TX *= tt;
      in_x[d] = true;
      t->xc = d;
    }
    break;
  }
  if (t->nx == 0) return ST_TOO_LARGE;
  // fewest load slots that cover the run
  int nvx = 8;
  while (nvx * V - V + 1 < TX) nvx *= 2;
  const int R1 = R;
  const int64_t tymax =
      std::min<int64_t>(tp.vt_nvy * V - V + 1, static_cast<int64_t>(R1) * (JV / (nvx / 8)));
  int64_t TY = 1;
  for (int k = 0; k < r; ++k) {
    const int d = p.perm[k];
    if (in_x[d]) break;
    if (k == 0 ? p.sB[d] != 1 : p.sB[d] != p.sB[p.perm[k - 1]] * p.n[p.perm[k - 1]]) break;
    if (TY * p.n[d] <= tymax) {
      t->yd[t->ny] = d;
      t->yt[t->ny++] = static_cast<int32_t>(p.n[d]);
      TY *= p.n[d];
      continue;
    }
    const int64_t c = tymax / TY;
    if (c >= 2) {
      const int64_t tt = cdiv(p.n[d], cdiv(p.n[d], c));
      t->yd[t->ny] = d;
      t->yt[t->ny++] = static_cast<int32_t>(tt);
      TY *= tt;
      t->yc = d;
    }
    break;
  }
  if (t->ny == 0) return ST_TOO_LARGE;
  int nvy = 8;
  while (nvy * V - V + 1 < TY) nvy *= 2;
  const int R2 = R;
  if (nvx / 8 > JV || nvy / 8 > JV) return ST_TOO_LARGE;
  if (cdiv(TY, R1) * (nvx / 8) > JV || cdiv(TX, R2) * (nvy / 8) > JV) return ST_TOO_LARGE;
  t->vlx = log2_slots(nvx);
  t->vly = log2_slots(nvy);
  t->TX = static_cast<int32_t>(TX);
  t->TY = static_cast<int32_t>(TY);
  t->RW = t->TX;
  t->WTY = t->TY;
  t->R1 = R1;
  t->J1 = static_cast<int32_t>(cdiv(TY, R1));
  t->R2 = R2;
  t->J2 = static_cast<int32_t>(cdiv(TX, R2));
  t->px = 1;
  t->py = 1;
  for (int i = 0; i + 1 < t->nx; ++i) t->px *= t->xt[i];
  for (int i = 0; i + 1 < t->ny; ++i) t->py *= t->yt[i];
  for (int i = 0; i < t->nx; ++i) tile_ext[t->xd[i]] = t->xt[i];
  for (int i = 0; i < t->ny; ++i) tile_ext[t->yd[i]] = t->yt[i];
  finish_grid(p, t, tile_ext, {t->xc, t->yc}, tp.grid_order);
  int64_t maxA = 0, maxB = 0;
  for (int i = 0; i < t->nx; ++i) {
    maxA += (t->xt[i] - 1) * p.sA[t->xd[i]];
    maxB += (t->xt[i] - 1) * p.sB[t->xd[i]];
  }
  for (int i = 0; i < t->ny; ++i) {
    maxA += (t->yt[i] - 1) * p.sA[t->yd[i]];
    maxB += (t->yt[i] - 1) * p.sB[t->yd[i]];
  }
  t->big_offsets = (maxA + V >= 0x7fffffffLL || maxB + V >= 0x7fffffffLL);
  const int off = t->big_offsets ? 8 : 4;
  auto a16 = [](int64_t x) { return static_cast<int32_t>((x + 15) & ~int64_t(15)); };
  t->tab2_off = a16(t->TY * off);
  t->thr_off = t->tab2_off + a16(t->TX * off);
  t->table_bytes = t->thr_off;
  finish_tables(p, t);
  // row pitch with the fewest bank conflicts (rows run from -(V-1), a row
  // holds the window slots' span)
  std::vector<int64_t> rowA, colB;
  vtile_maps(p, *t, &rowA, &colB);
  const int ld0 = nvx * V + V - 1;
  int best_ld = ld0, best_cost = 1 << 30;
  for (int ld = ld0; ld < ld0 + 128 / sz; ++ld) {
    const int c = vtile_bank_cost(*t, ld, sz, rowA, colB);
    if (c < best_cost) {
      best_cost = c;
      best_ld = ld;
    }
    if (c == 0) break;
  }
  t->LD = best_ld;
  const int64_t rows = static_cast<int64_t>(nvy) * V + V - 1;
  t->smem_bytes = a16(rows * t->LD * sz);
  if (t->smem_bytes > tp.smem_bytes * 3) return ST_TOO_LARGE;
  return t->num_tiles ? ST_OK : ST_TOO_LARGE;
}

// TMA tile (KIND_TTILE, ttile.cuh): tkx x tky boxes of 128 / sizeof(E)
// elements on each side, one grid level per tile position.
int choose_ttile(const HpttProblem &p, const TileParams &tp, int update, HpttTile *t) {
  if (!ttile_possible(p)) return ST_TOO_LARGE;
  const int sz = elem_bytes(p.dtype);
  const int box = 128 / sz;
  const int kx = tp.tt_kx, ky = tp.tt_ky;
  if (kx < 1 || ky < 1 || kx * ky > 8 || tp.tt < 1 || tp.tt > 4) return ST_TOO_LARGE;
  std::memset(t, 0, sizeof(*t));
  t->kind = KIND_TTILE;
  t->nt = 64 * kx * ky;
  if (tp.tt >= 2) {
    if (kx * ky > 4) return ST_TOO_LARGE;  // the persistent build's thread limit
    t->nt += 32;                           // the producer warp
  }
  t->W = 1;
  t->xc = t->yc = t->wc = -1;
  const int p0 = p.perm[0];
  t->nx = t->ny = 1;
  t->xd[0] = 0;
  t->yd[0] = p0;
  t->TX = kx * box;
  t->TY = ky * box;
  t->xt[0] = t->TX;
  t->yt[0] = t->TY;
  t->tkx = kx;
  t->tky = ky;
  t->ts = tp.tt >= 2 ? tp.tt : 0;
  int64_t tile_ext[HPTT_MAX_RANK];
  for (int d = 0; d < p.rank; ++d) tile_ext[d] = 1;
  tile_ext[0] = t->TX;
  tile_ext[p0] = t->TY;
  finish_grid(p, t, tile_ext, {0, p0}, tp.grid_order);
  // one CTA per tile: A's and B's boxes, the mbarrier (16 bytes at the
  // base) and the slack that aligns the boxes to the 128-byte swizzle's
  // 1024-byte pattern; persistent CTAs: ts stages of A's boxes (and B's when
  // B is read), three output buffers of boxes, a 256-byte header (mbarriers
  // and tile origins) and the same slack
  const int kb = kx * ky * box * 128;
  t->smem_bytes = t->ts ? t->ts * kb * (update ? 2 : 1) + 3 * kb + 1024 + 256
                        : 2 * kb + 1024 + 16;
  if (t->smem_bytes > 227 * 1024) return ST_TOO_LARGE;  // sm_100a's per-CTA limit
  t->tab2_off = 16;
  t->thr_off = 16;
  t->table_bytes = 16;
  return t->num_tiles ? ST_OK : ST_TOO_LARGE;
}

}  // namespace

bool ttile_possible(const HpttProblem &p) {
  const int sz = elem_bytes(p.dtype);
  if ((sz != 4 && sz != 8) || p.rank < 2 || p.rank > 5 || p.perm[0] == 0) return false;
  for (int d = 0; d < p.rank; ++d) {
    // TMA box coordinates are signed 32-bit: a tile's origin plus its box
    // offsets (under 2^10) must stay positive, so extents stay at or below
    // 2^30
    if (p.n[d] < 1 || p.n[d] > (int64_t(1) << 30)) return false;
    if (d > 0 && ((p.sA[d] * sz) % 16 != 0 || p.sA[d] * sz >= (int64_t(1) << 40))) return false;
    if (d != p.perm[0] && ((p.sB[d] * sz) % 16 != 0 || p.sB[d] * sz >= (int64_t(1) << 40)))
      return false;
  }
  return p.sA[0] == 1 && p.sB[p.perm[0]] == 1;
}

int ttile_map_params(const HpttProblem &p, const HpttTile &t, int side, TtileMapParams *out) {
  if (t.kind != KIND_TTILE || !ttile_possible(p)) return ST_TOO_LARGE;
  const int sz = elem_bytes(p.dtype);
  const uint32_t box = 128 / sz;
  out->rank = p.rank;
  out->elem_bytes = sz;
  for (int k = 0; k < p.rank; ++k) {
    const int d = side == 0 ? k : p.perm[k];  // input dim of this map dim
    out->dims[k] = static_cast<uint64_t>(p.n[d]);
    out->stride_bytes[k] = static_cast<uint64_t>(side == 0 ? p.sA[d] : p.sB[d]) * sz;
    out->box[k] = d == 0 ? box : (d == p.perm[0] ? box : 1u);
  }
  return ST_OK;
}

bool vtile_possible(const HpttProblem &p) {
  const int sz = elem_bytes(p.dtype);
  return (sz == 4 || sz == 8) && p.rank >= 2 && p.perm[0] != 0;
}

void vtile_maps(const HpttProblem &p, const HpttTile &t, std::vector<int64_t> *rowA,
                std::vector<int64_t> *colB) {
  rowA->assign(static_cast<size_t>(t.TY), 0);
  colB->assign(static_cast<size_t>(t.TX), 0);
  int c = 0;
  for (int y = 0; y < t.TY; ++y)
    (*rowA)[y] = side_offset(y, t.ny, t.yd, t.yt, p.sA, -1, &c);
  for (int x = 0; x < t.TX; ++x)
    (*colB)[x] = side_offset(x, t.nx, t.xd, t.xt, p.sB, -1, &c);
}

int choose_tile(const HpttProblem &p, const TileParams &tp, int update, HpttTile *t) {
  // the shapes are the same with and without the B read (only the vector
  // tile's early B reads depend on it)
  const int sz = elem_bytes(p.dtype);
  const int r = p.rank;
  const bool common = p.perm[0] == 0;
  if (r == 1 || (common && p.n[0] * sz >= tp.rows_min_bytes))
    return choose_rows(p, tp, t);
  if (common && p.n[0] > tp.nt / 2) return choose_rows(p, tp, t);
  if (tp.tt && ttile_possible(p) && choose_ttile(p, tp, update, t) == ST_OK) return ST_OK;
  if (tp.vt && vtile_possible(p) && choose_vtile(p, tp, update, t) == ST_OK) return ST_OK;

  std::memset(t, 0, sizeof(*t));
  t->kind = KIND_TILE;
  t->nt = tp.nt;
  t->vec = 1;
  t->xc = t->yc = t->wc = -1;
  const int64_t W = common ? p.n[0] : 1;
  const int si = common ? 1 : 0, so = common ? 1 : 0;
  const int64_t target = std::max<int64_t>(4, tp.run_bytes / sz);
  bool in_tile[HPTT_MAX_RANK] = {false};
  if (common) in_tile[0] = true;

  Side X, Y;
  // X: input-order dims (stopping at the output's leading dim, or skipping
  // dims Y already holds when Y is chosen first); Y: output-order dims.
  auto pick_x = [&]() {
    int64_t prod = W;
    for (int d = si; d < r; ++d) {
      if (in_tile[d]) {
        if (tp.y_first) continue;
        break;
      }
      if (!tp.y_first && d == p.perm[so]) break;
      const int64_t cap = tp.nt / prod;
      const int64_t tt = std::min({p.n[d], cdiv(target, prod), cap});
      if (tt < 1) break;
      X.d.push_back(d);
      X.t.push_back(tt);
      in_tile[d] = true;
      prod *= tt;
      if (tt < p.n[d] || prod >= target) break;
    }
  };
  auto pick_y = [&]() {
    int64_t prod = W;
    for (int k = so; k < r; ++k) {
      const int d = p.perm[k];
      if (in_tile[d]) break;
      const int64_t cap = tp.nt / prod;
      const int64_t tt = std::min({p.n[d], cdiv(target, prod), cap});
      if (tt < 1) break;
      Y.d.push_back(d);
      Y.t.push_back(tt);
      in_tile[d] = true;
      prod *= tt;
      if (tt < p.n[d] || prod >= target) break;
    }
  };
  if (tp.y_first) {
    pick_y();
    pick_x();
  } else {
    pick_x();
    pick_y();
  }
  // shrink until the shape fits the thread mapping (the larger side first)
  for (int guard = 0; guard < 4096 && !shape_ok(tp, W, X, Y, sz); ++guard) {
    Side *S = (X.prod() >= Y.prod()) ? &X : &Y;
    if (S->d.empty()) S = (S == &X) ? &Y : &X;
    if (S->d.empty()) break;
    int64_t &tt = S->t.back();
    if (tt > 1) {
      tt = std::max<int64_t>(1, (tt * 3) / 4);
    } else {
      in_tile[S->d.back()] = false;
      S->d.pop_back();
      S->t.pop_back();
    }
  }
  // grow the tile until it holds vmin bytes
  const int64_t vmin = std::max<int64_t>(1, tp.vmin_bytes / sz);
  auto vol = [&]() { return W * X.prod() * Y.prod(); };
  auto next_in = [&](const Side &S, bool output_order) -> int {
    // next dim to add after a full last dim
    if (output_order) {
      for (int k = so; k < r; ++k) {
        const int d = p.perm[k];
        if (!in_tile[d]) return d;
      }
      return -1;
    }
    for (int d = si; d < r; ++d)
      if (!in_tile[d]) return d;
    (void)S;
    return -1;
  };
  for (int iter = 0; iter < 64 && vol() < vmin; ++iter) {
    bool grown = false;
    // the side with the shorter run first
    const bool x_first = X.prod() <= Y.prod();
    for (int pass = 0; pass < 4 && !grown; ++pass) {
      const bool onX = (pass % 2 == 0) ? x_first : !x_first;
      Side &S = onX ? X : Y;
      if (pass < 2) {
        // enlarge the chunked last dim
        if (S.d.empty()) continue;
        const int d = S.d.back();
        int64_t &tt = S.t.back();
        if (tt >= p.n[d]) continue;
        const int64_t old = tt;
        const int64_t want = std::min<int64_t>(p.n[d], std::max<int64_t>(old + 1, old * 2));
        tt = want;
        while (tt > old && !shape_ok(tp, W, X, Y, sz)) --tt;
        if (tt > old) grown = true; else tt = old;
      } else {
        if (!S.d.empty() && S.t.back() < p.n[S.d.back()]) continue;
        const int d = next_in(S, !onX);
        if (d < 0) continue;
        S.d.push_back(d);
        S.t.push_back(1);
        in_tile[d] = true;
        int64_t &tt = S.t.back();
        const int64_t want = std::min<int64_t>(p.n[d], cdiv(vmin, vol()));
        tt = std::max<int64_t>(1, want);
        while (tt > 1 && !shape_ok(tp, W, X, Y, sz)) --tt;
        if (tt > 1 && shape_ok(tp, W, X, Y, sz)) {
          grown = true;
        } else {
          S.d.pop_back();
          S.t.pop_back();
          in_tile[d] = false;
        }
      }
    }
    if (!grown) break;
  }
  // Chunked last dims: take the whole extent when it is only a little larger
  // than the chunk, else split it into equal chunks, so edge tiles are not
  // mostly empty (72 = 64 + 8 becomes 2 x 36).
  for (Side *S : {&X, &Y}) {
    if (S->d.empty()) continue;
    const int64_t n = p.n[S->d.back()];
    int64_t &tt = S->t.back();
    if (tt >= n) continue;
    const int64_t old = tt;
    if (2 * n <= 3 * tt) {
      tt = n;
      if (shape_ok(tp, W, X, Y, sz)) continue;
      tt = old;
    }
    tt = cdiv(n, cdiv(n, old));
  }
  // Whole-extent option (autotuner knob): one side takes its full single-dim
  // extent, the other shrinks until the tile fits, in whole sectors when it
  // can.
  if (tp.full_side && X.d.size() == 1 && Y.d.size() == 1) {
    Side &F = tp.full_side == 1 ? X : Y;
    Side &O = tp.full_side == 1 ? Y : X;
    const int64_t nF = p.n[F.d.back()];
    if (F.t.back() < nF) {
      const int64_t oldF = F.t.back(), oldO = O.t.back();
      F.t.back() = nF;
      const int64_t sector = std::max<int64_t>(1, 32 / sz);
      int64_t &to = O.t.back();
      while (to > 1 && !shape_ok(tp, W, X, Y, sz)) {
        // largest multiple of a sector below the current extent, else -1
        const int64_t down = (to - 1) / sector * sector;
        to = down >= sector ? down : to - 1;
      }
      if (!shape_ok(tp, W, X, Y, sz) || to * sz < 32) {
        F.t.back() = oldF;
        O.t.back() = oldO;
      }
    }
  }
  // Single-dim sides: round a chunked extent to a multiple of the threads
  // per pass on its side (TY to R1, TX to R2), so every thread of an
  // interior tile has the same iteration count and the kernel's predicate-
  // free path applies ("even" tiles).
  if (X.d.size() == 1 && Y.d.size() == 1) {
    for (int round = 0; round < 2; ++round) {
      for (int side = 0; side < 2; ++side) {
        Side &S = side == 0 ? Y : X;
        const int64_t n = p.n[S.d.back()];
        int64_t &tt = S.t.back();
        if (tt >= n) continue;
        const int64_t other = side == 0 ? W * X.prod() : W * Y.prod();
        const int64_t R = other > 0 ? tp.nt / other : 0;
        if (R <= 1 || tt % R == 0) continue;
        const int64_t old = tt;
        tt = std::min<int64_t>(n, cdiv(old, R) * R);
        if (tt < n && shape_ok(tp, W, X, Y, sz)) continue;
        tt = (old / R) * R;
        if (tt >= R && shape_ok(tp, W, X, Y, sz)) continue;
        tt = old;
      }
    }
  }
  if (!shape_ok(tp, W, X, Y, sz)) return ST_TOO_LARGE;
  // A trailing dim with tile extent 1 adds nothing to the tile (the grid
  // steps through it either way) but would keep the side off the single-dim
  // kernel path: drop it.
  for (Side *S : {&X, &Y}) {
    while (S->d.size() > 1 && S->t.back() == 1) {
      in_tile[S->d.back()] = false;
      S->d.pop_back();
      S->t.pop_back();
    }
  }

  t->W = static_cast<int32_t>(W);
  t->nx = static_cast<int32_t>(X.d.size());
  t->ny = static_cast<int32_t>(Y.d.size());
  int64_t tile_ext[HPTT_MAX_RANK];
  for (int d = 0; d < r; ++d) tile_ext[d] = 1;
  if (common) tile_ext[0] = W;
  for (int i = 0; i < t->nx; ++i) {
    t->xd[i] = X.d[i];
    t->xt[i] = static_cast<int32_t>(X.t[i]);
    tile_ext[X.d[i]] = X.t[i];
  }
  for (int i = 0; i < t->ny; ++i) {
    t->yd[i] = Y.d[i];
    t->yt[i] = static_cast<int32_t>(Y.t[i]);
    tile_ext[Y.d[i]] = Y.t[i];
  }
  if (t->nx && X.t.back() < p.n[X.d.back()]) t->xc = X.d.back();
  if (t->ny && Y.t.back() < p.n[Y.d.back()]) t->yc = Y.d.back();
  t->TX = static_cast<int32_t>(X.prod());
  t->px = 1;
  t->py = 1;
  for (int i = 0; i + 1 < t->nx; ++i) t->px *= t->xt[i];
  for (int i = 0; i + 1 < t->ny; ++i) t->py *= t->yt[i];
  t->TY = static_cast<int32_t>(Y.prod());
  t->RW = static_cast<int32_t>(W * t->TX);
  t->WTY = static_cast<int32_t>(W * t->TY);
  t->R1 = t->nt / t->RW;
  t->J1 = static_cast<int32_t>(cdiv(t->TY, t->R1));
  t->R2 = t->nt / t->WTY;
  t->J2 = static_cast<int32_t>(cdiv(t->TX, t->R2));
  t->even = (t->TY == t->R1 * t->J1 && t->TX == t->R2 * t->J2) ? 1 : 0;
  // row pitch with the fewest shared-memory bank conflicts
  TileMaps maps;
  tile_maps(p, *t, &maps);
  int best_ld = t->RW, best_cost = 1 << 30;
  const int span = std::max(1, 128 / sz);
  for (int ld = t->RW; ld < t->RW + span; ++ld) {
    const int c = bank_cost(*t, ld, sz, maps);
    if (c < best_cost) {
      best_cost = c;
      best_ld = ld;
    }
    if (c == 0) break;
  }
  t->LD = best_ld;
  finish_grid(p, t, tile_ext, {t->xc, t->yc}, tp.grid_order);

  int64_t maxA = 0, maxB = 0;
  if (common) {
    maxA += (W - 1) * p.sA[0];
    maxB += (W - 1) * p.sB[0];
  }
  for (int i = 0; i < t->nx; ++i) {
    maxA += (t->xt[i] - 1) * p.sA[t->xd[i]];
    maxB += (t->xt[i] - 1) * p.sB[t->xd[i]];
  }
  for (int i = 0; i < t->ny; ++i) {
    maxA += (t->yt[i] - 1) * p.sA[t->yd[i]];
    maxB += (t->yt[i] - 1) * p.sB[t->yd[i]];
  }
  t->big_offsets = (maxA >= 0x7fffffffLL || maxB >= 0x7fffffffLL);
  const int off = t->big_offsets ? 8 : 4;
  t->smem_bytes = (t->TY * t->LD * sz + 15) & ~15;
  auto a16 = [](int x) { return (x + 15) & ~15; };
  const int ent = 2 * off;  // sizeof(HpttTabEnt<OffT>)
  t->tab2_off = a16(t->TY * ent);
  t->thr_off = t->tab2_off + a16(t->TX * ent);
  t->table_bytes = t->thr_off + t->nt * static_cast<int>(sizeof(HpttThr));
  finish_tables(p, t);
  if (!tp.walk) {
    std::memset(&t->wx, 0, sizeof(t->wx));
    std::memset(&t->wy, 0, sizeof(t->wy));
  }
  t->upd_exact = tp.upd_exact ? 1 : 0;
  return t->num_tiles ? ST_OK : ST_TOO_LARGE;
}

std::string describe(const HpttProblem &p, const HpttTile &t) {
  static const char *names[] = {"float", "double", "complex float", "complex double"};
  std::ostringstream os;
  os << "dtype: " << names[p.dtype & 3] << "\n";
  os << "fused rank: " << p.rank << "\n  extents (input order):";
  for (int d = 0; d < p.rank; ++d) os << " " << p.n[d];
  os << "\n  perm (output dim -> input dim):";
  for (int k = 0; k < p.rank; ++k) os << " " << p.perm[k];
  os << "\n  strides A:";
  for (int d = 0; d < p.rank; ++d) os << " " << p.sA[d];
  os << "\n  strides B:";
  for (int d = 0; d < p.rank; ++d) os << " " << p.sB[d];
  os << "\nkernel: "
     << (t.kind == KIND_TILE    ? "tile (shared-memory transpose)"
         : t.kind == KIND_VTILE ? "vector tile (16-byte windows, shared-memory transpose)"
         : t.kind == KIND_TTILE ? "TMA tile (tensor-map box loads and stores, shared-memory transpose)"
                                : "rows (shared stride-1)")
     << ", " << t.nt << " threads/CTA";
  if (t.kind == KIND_ROWS) os << ", vector " << t.vec;
  if (t.kind == KIND_TTILE) {
    os << ", boxes " << t.tkx << " x " << t.tky;
    if (t.ts) os << ", persistent, " << t.ts << " stages";
  }
  if (t.kind == KIND_VTILE)
    os << ", slots " << (8 << t.vlx) << " x " << (8 << t.vly) << ", J " << t.J1 << "/" << t.J2
       << ", " << t.vj << " vectors/thread" << (t.vpre ? ", B read first" : "");
  os << "\n  tile W=" << t.W << " X{";
  for (int i = 0; i < t.nx; ++i) os << (i ? "," : "") << t.xd[i] << ":" << t.xt[i];
  os << "} Y{";
  for (int i = 0; i < t.ny; ++i) os << (i ? "," : "") << t.yd[i] << ":" << t.yt[i];
  os << "} TX=" << t.TX << " TY=" << t.TY << " LD=" << t.LD;
  if (t.wx.e0 || t.wy.e0)
    os << " walked:" << (t.wx.e0 ? " X" : "") << (t.wy.e0 ? " Y" : "");
  os << "\n  tiles: " << t.num_tiles << ", smem/CTA: " << t.smem_bytes
     << " B, tables: " << t.table_bytes << " B\n";
  return os.str();
}

}  // namespace hptt_b200
