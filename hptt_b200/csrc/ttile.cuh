// sm_100a tensor-memory-accelerator tile: B = alpha * A(perm) + beta * B with
// the global side of both phases done by TMA (cp.async.bulk.tensor).
//
// Shape (KIND_TTILE, planned by choose_tile): fused rank <= 5, 4- or 8-byte
// elements, every stride of A and B other than the unit one a multiple of 16
// bytes, and a true transpose (input dim 0 is not output dim 0).  A tile is
// tkx x tky boxes of BX x BY elements, BX along input dim 0 and BY along the
// output's leading dim p0 (input dim perm[0]); a box row is 128 bytes on both
// sides (BX = BY = 128 / sizeof(E)).
//
// Per CTA (64 threads per box):
//   1. one thread arms an mbarrier with the tile's byte count and issues one
//      TMA load per box of A -- and, when B is read, of B -- into shared
//      memory with the 128-byte swizzle (16-byte chunk c of box row r sits
//      at chunk c ^ (r & 7));
//   2. every thread waits for the mbarrier (a bounded wait: see
//      ttile_wait), then each box's 64 threads transpose it: a thread reads
//      an m x m micro-block (m = 16 / sizeof(E)) as m 16-byte rows of the A
//      box, transposes it in registers, and writes m 16-byte rows of the
//      B-side box (combining them with B's old values when B is read).
//      Micro-block (xb, yb) = (l, (l + p) & 7) for thread t = 8 p + l: with
//      the swizzle, every 8-thread phase of every 16-byte shared access then
//      touches 8 distinct chunks, so no access has a bank conflict;
//   3. after a proxy fence and a barrier, one thread issues one TMA store per
//      box and waits until the stores have read shared memory.
// Persistent form (HpttTile::ts = S stages): a grid of resident CTAs walks
// the tiles (tile blockIdx.x + i gridDim.x), warp-specialised.  A producer
// lane keeps the CTA's next S tiles' loads in flight in a ring of S stages,
// each with a "full" mbarrier (armed with the tile's bytes; phase parity
// (i / S) & 1 for the CTA's i-th tile) and an "empty" one the consumers
// arrive on once they have read the stage.  The consumer threads (64 per
// box) transpose into one of three output buffers, which the TMA stores read
// while the next tiles are transposed: before the consumers' barrier of
// tile i, their thread 0 waits until at most one store group is still
// reading shared memory (cp.async.bulk.wait_group.read 1), so the buffer of
// tile i - 2 is free for tile i + 1.
//
// TMA clips at the tensor's edges (loads fill zeros outside, stores skip
// them), so edge tiles need no code of their own.  The innermost coordinate
// of every load and store is a multiple of BX or BY (128 bytes), which TMA
// requires; nothing else needs alignment.
//
// The reference moves whole 256-bit rows through registers
// (src/arch/avx2/kernel_trans_avx2.cc:21-467); here whole box rows move
// between HBM and shared memory without any thread issuing an address.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "desc.h"
#include "kernels.cuh"
#include "ops.cuh"

namespace hptt_b200 {
namespace dev {

// Coordinates of tile `tile`'s origin along every input dim (dims outside
// the grid stay 0): the grid levels of HpttTile, each dim's coordinate the
// level's position times its step.
HPTT_HD inline void ttile_coords(const HpttTile &T, uint32_t tile, int32_t *coord) {
  for (int d = 0; d < 5; ++d) coord[d] = 0;
  uint32_t rem = tile;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int g = 0; g < HPTT_MAX_RANK; ++g) {
    if (g < T.ng) {
      const uint32_t q = T.gmul[g] ? (umulhi32(rem, T.gmul[g]) >> T.gshr[g]) : rem;
      const uint32_t c = rem - q * T.gcnt[g];
      rem = q;
      const int d = T.gd[g];
      if (d < 5) coord[d] = static_cast<int32_t>(c) * T.gstep[g];
    }
  }
}

// Byte offset of 16-byte chunk `chunk` of box row `row` under the 128-byte
// swizzle (rows of 128 bytes, the buffer 1024-byte aligned).
HPTT_HD inline uint32_t ttile_swz(uint32_t row, uint32_t chunk) {
  return row * 128u + ((chunk ^ (row & 7u)) << 4);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// TMA load of one box into shared memory, completing on mbarrier `bar`.
__device__ __forceinline__ void ttile_load(const void *tmap, uint32_t dst, uint32_t bar,
                                           int rank, const int32_t *c) {
  const uint64_t m = reinterpret_cast<uint64_t>(tmap);
  switch (rank) {
    case 2:
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]), "r"(bar)
          : "memory");
      break;
    case 3:
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]),
          "r"(c[2]), "r"(bar)
          : "memory");
      break;
    case 4:
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]),
          "r"(c[2]), "r"(c[3]), "r"(bar)
          : "memory");
      break;
    default:
      asm volatile(
          "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst), "l"(m), "r"(c[0]), "r"(c[1]),
          "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(bar)
          : "memory");
      break;
  }
}

// TMA store of one box from shared memory (bulk group of this thread).
__device__ __forceinline__ void ttile_store(const void *tmap, uint32_t src, int rank,
                                            const int32_t *c) {
  const uint64_t m = reinterpret_cast<uint64_t>(tmap);
  switch (rank) {
    case 2:
      asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                   ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(src)
                   : "memory");
      break;
    case 3:
      asm volatile(
          "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
          ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(src)
          : "memory");
      break;
    case 4:
      asm volatile(
          "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
          ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(src)
          : "memory");
      break;
    default:
      asm volatile(
          "cp.async.bulk.tensor.5d.global.shared::cta.bulk_group"
          " [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]),
          "r"(c[3]), "r"(c[4]), "r"(src)
          : "memory");
      break;
  }
}

// Wait for the phase of mbarrier `bar` with parity `parity` to complete, at
// most `limit` polls (each poll may suspend the thread for a short,
// hardware-chosen time).  Returns false when the limit ran out.
__device__ __forceinline__ bool ttile_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
  for (uint32_t k = 0; k < limit; ++k) {
    uint32_t done = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace dev
}  // namespace hptt_b200
