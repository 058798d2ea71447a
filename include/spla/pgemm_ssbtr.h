/* pgemm_ssb restricted to a triangle of C. Elements of C outside the triangle
 * selected by cFillMode may or may not be computed: this library skips the
 * tiles of C that lie entirely outside it and leaves those elements unchanged.
 * Replaces include/spla/pgemm_ssbtr.h:94-128. */
#ifndef SPLA_PGEMM_SSBTR_H
#define SPLA_PGEMM_SSBTR_H
#include "spla/config.h"
#include "spla/context.h"
#include "spla/errors.h"
#include "spla/matrix_distribution.h"

#ifdef __cplusplus
extern "C" {
#endif

/* pgemm_ssbtr.h:94 */
SPLA_EXPORT SplaError spla_psgemm_ssbtr(int m, int n, int kLocal, SplaOperation opA, float alpha,
                                        const float *A, int lda, const float *B, int ldb,
                                        float beta, float *C, int ldc, int cRowOffset,
                                        int cColOffset, SplaFillMode cFillMode,
                                        SplaMatrixDistribution distC, SplaContext ctx);
/* pgemm_ssbtr.h:104 */
SPLA_EXPORT SplaError spla_pdgemm_ssbtr(int m, int n, int kLocal, SplaOperation opA, double alpha,
                                        const double *A, int lda, const double *B, int ldb,
                                        double beta, double *C, int ldc, int cRowOffset,
                                        int cColOffset, SplaFillMode cFillMode,
                                        SplaMatrixDistribution distC, SplaContext ctx);
/* pgemm_ssbtr.h:114 */
SPLA_EXPORT SplaError spla_pcgemm_ssbtr(int m, int n, int kLocal, SplaOperation opA,
                                        const void *alpha, const void *A, int lda, const void *B,
                                        int ldb, const void *beta, void *C, int ldc, int cRowOffset,
                                        int cColOffset, SplaFillMode cFillMode,
                                        SplaMatrixDistribution distC, SplaContext ctx);
/* pgemm_ssbtr.h:124 */
SPLA_EXPORT SplaError spla_pzgemm_ssbtr(int m, int n, int kLocal, SplaOperation opA,
                                        const void *alpha, const void *A, int lda, const void *B,
                                        int ldb, const void *beta, void *C, int ldc, int cRowOffset,
                                        int cColOffset, SplaFillMode cFillMode,
                                        SplaMatrixDistribution distC, SplaContext ctx);
#ifdef __cplusplus
}
#endif
#endif
