/*
 * CPU oracle for B = alpha * A(perm) + beta * B.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as a checker or a timed CPU baseline.  The
 * product (libhptt_cuda.so) never links or calls it.
 *
 * Parity pinning: the restatement is checked bit-for-bit against the
 * reference's own CPU plan (built from the reference sources by
 * oracle/Makefile into oracle/_ref/) on every case where that plan is
 * correct, and against the committed fixtures in tests/golden/ that were
 * produced by that build.
 */
#ifndef HPTT_ORACLE_H_
#define HPTT_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element types, same numbering as include/hptt_cuda.h. */
enum { ORACLE_F32 = 0, ORACLE_F64 = 1, ORACLE_C64 = 2, ORACLE_C128 = 3 };

/*
 * Naive transpose.  rank >= 1; in_size/perm have `rank` entries;
 * in_outer/out_outer may be NULL (then equal to the inner sizes; out_outer is
 * indexed by OUTPUT dimension).  alpha/beta point to 2 doubles (re, im); for
 * real element types only [0] is used.  complex_scalars != 0 selects the
 * complex-scalar extension for C64/C128; otherwise alpha[0]/beta[0] are real
 * scalars applied componentwise, as in the reference.
 * Returns 0 on success, -1 on bad arguments.
 */
int hptt_oracle_trans(int dtype, int rank, const uint32_t *in_size,
                      const uint32_t *perm, const uint32_t *in_outer,
                      const uint32_t *out_outer, const double *alpha,
                      const double *beta, int complex_scalars,
                      const void *in, void *out, int num_threads);

/* 1 when B is read (|beta| >= 1e-16), following the reference rule. */
int hptt_oracle_update(int dtype, const double *beta, int complex_scalars);

#ifdef __cplusplus
}
#endif

#endif
