// Tensor contraction by transpose - GEMM - transpose (TTGT).
//
//   C[lc] = alpha * sum_{k labels} A[la] * B[lb] + beta * C[lc]
//
// Every label is one of: M (in A and C), N (in B and C), K (in A and B,
// summed) or BATCH (in A, B and C).  A is staged as the column-major matrix
// [M, K] or [K, M] per batch, B as [K, N] or [N, K], the GEMM writes C-hat as
// [M, N] or (operands swapped) [N, M], and the output transpose applies alpha
// and beta while it moves C-hat into C's layout.  An operand already in a
// staged layout is used in place.  The host-only analysis below picks label
// orders and layouts that move the fewest bytes.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "desc.h"

namespace hptt_b200 {

struct ContractLayout {
  int dtype = 0;
  int ra = 0, rb = 0, rc = 0;
  int32_t la[HPTT_MAX_RANK], lb[HPTT_MAX_RANK], lc[HPTT_MAX_RANK];
  uint32_t sa[HPTT_MAX_RANK], sb[HPTT_MAX_RANK], sc[HPTT_MAX_RANK];

  // label lists of each class, in the chosen order
  int nm = 0, nn = 0, nk = 0, nbat = 0;
  int32_t ml[HPTT_MAX_RANK], nl[HPTT_MAX_RANK], kl[HPTT_MAX_RANK], bl[HPTT_MAX_RANK];

  int a_km = 0;  // A-hat is [K, M, BATCH] (else [M, K, BATCH])
  int b_nk = 0;  // B-hat is [N, K, BATCH] (else [K, N, BATCH])
  int swap = 0;  // the GEMM writes C-hat as [N, M, BATCH] (else [M, N, BATCH])
  int tr_a = 0, tr_b = 0, tr_c = 0;  // which transposes run

  uint64_t m = 1, n = 1, k = 1, batch = 1;
  uint64_t elems_a = 1, elems_b = 1, elems_c = 1;

  // transposes: input sizes (the source's own order) and perm
  uint32_t pa_perm[HPTT_MAX_RANK], pb_perm[HPTT_MAX_RANK], pc_perm[HPTT_MAX_RANK];
  uint32_t chat_size[HPTT_MAX_RANK];  // C-hat extents in its label order

  // workspace: A-hat, B-hat, C-hat (when transposed) and the GEMM library's
  // own workspace, each 256-byte aligned
  uint64_t off_a = 0, off_b = 0, off_c = 0, off_blas = 0, ws_bytes = 0;
  uint64_t moved_bytes = 0;  // transpose bytes per exec (2 * elements * size each)
};

// Bytes reserved for the GEMM library's workspace inside the contraction
// workspace.
constexpr uint64_t kBlasWorkspaceBytes = 32ull << 20;

// Validate labels and sizes and choose the layout.  ra/rb in 1..8, rc in
// 0..8.  Returns ST_OK, ST_BAD_DTYPE, ST_BAD_RANK, ST_BAD_SIZE_VALUE,
// ST_LABELS or ST_TOO_LARGE (a GEMM extent above 2^31 - 1).
int contract_analyze(int dtype, int ra, const uint32_t *sa, const int32_t *la, int rb,
                     const uint32_t *sb, const int32_t *lb, int rc, const int32_t *lc,
                     ContractLayout *out);

// Readable summary of a layout.
void contract_describe(const ContractLayout &L, char *buf, size_t len);

}  // namespace hptt_b200
