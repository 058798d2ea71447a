/* Stripe x stripe -> block:  C <- alpha * op(A) * B + beta * C, op(A) = A^T or A^H.
 * A (kLocal x m, lda >= kLocal) and B (kLocal x n, ldb >= kLocal) are column-major
 * stripes of the long dimension k; C is the m x n sub-block of the distributed C
 * starting at (cRowOffset, cColOffset). Complex arguments are interleaved (re, im)
 * pairs; alpha/beta point to one such pair. Replaces include/spla/pgemm_ssb.h:88-121. */
#ifndef SPLA_PGEMM_SSB_H
#define SPLA_PGEMM_SSB_H
#include "spla/config.h"
#include "spla/context.h"
#include "spla/errors.h"
#include "spla/matrix_distribution.h"

#ifdef __cplusplus
extern "C" {
#endif

/* pgemm_ssb.h:88 */
SPLA_EXPORT SplaError spla_psgemm_ssb(int m, int n, int kLocal, SplaOperation opA, float alpha,
                                      const float *A, int lda, const float *B, int ldb, float beta,
                                      float *C, int ldc, int cRowOffset, int cColOffset,
                                      SplaMatrixDistribution distC, SplaContext ctx);
/* pgemm_ssb.h:97 */
SPLA_EXPORT SplaError spla_pdgemm_ssb(int m, int n, int kLocal, SplaOperation opA, double alpha,
                                      const double *A, int lda, const double *B, int ldb,
                                      double beta, double *C, int ldc, int cRowOffset,
                                      int cColOffset, SplaMatrixDistribution distC,
                                      SplaContext ctx);
/* pgemm_ssb.h:107 */
SPLA_EXPORT SplaError spla_pcgemm_ssb(int m, int n, int kLocal, SplaOperation opA,
                                      const void *alpha, const void *A, int lda, const void *B,
                                      int ldb, const void *beta, void *C, int ldc, int cRowOffset,
                                      int cColOffset, SplaMatrixDistribution distC,
                                      SplaContext ctx);
/* pgemm_ssb.h:117 */
SPLA_EXPORT SplaError spla_pzgemm_ssb(int m, int n, int kLocal, SplaOperation opA,
                                      const void *alpha, const void *A, int lda, const void *B,
                                      int ldb, const void *beta, void *C, int ldc, int cRowOffset,
                                      int cColOffset, SplaMatrixDistribution distC,
                                      SplaContext ctx);
#ifdef __cplusplus
}
#endif
#endif
