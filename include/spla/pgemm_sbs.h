/* Stripe x block -> stripe:  C <- alpha * A * B + beta * C.
 * A (mLocal x k, lda >= mLocal) and C (mLocal x n, ldc >= mLocal) are row stripes;
 * B is the k x n sub-block of the distributed B at (bRowOffset, bColOffset).
 * Note that beta follows distB. Replaces include/spla/pgemm_sbs.h:85-115. */
#ifndef SPLA_PGEMM_SBS_H
#define SPLA_PGEMM_SBS_H
#include "spla/config.h"
#include "spla/context.h"
#include "spla/errors.h"
#include "spla/matrix_distribution.h"

#ifdef __cplusplus
extern "C" {
#endif

/* pgemm_sbs.h:85 */
SPLA_EXPORT SplaError spla_psgemm_sbs(int mLocal, int n, int k, float alpha, const float *A,
                                      int lda, const float *B, int ldb, int bRowOffset,
                                      int bColOffset, SplaMatrixDistribution distB, float beta,
                                      float *C, int ldc, SplaContext ctx);
/* pgemm_sbs.h:94 */
SPLA_EXPORT SplaError spla_pdgemm_sbs(int mLocal, int n, int k, double alpha, const double *A,
                                      int lda, const double *B, int ldb, int bRowOffset,
                                      int bColOffset, SplaMatrixDistribution distB, double beta,
                                      double *C, int ldc, SplaContext ctx);
/* pgemm_sbs.h:103 */
SPLA_EXPORT SplaError spla_pcgemm_sbs(int mLocal, int n, int k, const void *alpha, const void *A,
                                      int lda, const void *B, int ldb, int bRowOffset,
                                      int bColOffset, SplaMatrixDistribution distB,
                                      const void *beta, void *C, int ldc, SplaContext ctx);
/* pgemm_sbs.h:112 */
SPLA_EXPORT SplaError spla_pzgemm_sbs(int mLocal, int n, int k, const void *alpha, const void *A,
                                      int lda, const void *B, int ldb, int bRowOffset,
                                      int bColOffset, SplaMatrixDistribution distB,
                                      const void *beta, void *C, int ldc, SplaContext ctx);
#ifdef __cplusplus
}
#endif
#endif
