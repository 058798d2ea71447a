/* Local GEMM  C <- alpha * op(A) * op(B) + beta * C  (column-major, op in N/T/C),
 * with any mix of host and device pointers. Replaces include/spla/gemm.h:65-94. */
#ifndef SPLA_GEMM_H
#define SPLA_GEMM_H
#include "spla/config.h"
#include "spla/context.h"
#include "spla/errors.h"

#ifdef __cplusplus
extern "C" {
#endif

/* gemm.h:65 */
SPLA_EXPORT SplaError spla_sgemm(SplaOperation opA, SplaOperation opB, int m, int n, int k,
                                 float alpha, const float *A, int lda, const float *B, int ldb,
                                 float beta, float *C, int ldc, SplaContext ctx);
/* gemm.h:74 */
SPLA_EXPORT SplaError spla_dgemm(SplaOperation opA, SplaOperation opB, int m, int n, int k,
                                 double alpha, const double *A, int lda, const double *B, int ldb,
                                 double beta, double *C, int ldc, SplaContext ctx);
/* gemm.h:83 */
SPLA_EXPORT SplaError spla_cgemm(SplaOperation opA, SplaOperation opB, int m, int n, int k,
                                 const void *alpha, const void *A, int lda, const void *B, int ldb,
                                 const void *beta, void *C, int ldc, SplaContext ctx);
/* gemm.h:92 */
SPLA_EXPORT SplaError spla_zgemm(SplaOperation opA, SplaOperation opB, int m, int n, int k,
                                 const void *alpha, const void *A, int lda, const void *B, int ldb,
                                 const void *beta, void *C, int ldc, SplaContext ctx);
#ifdef __cplusplus
}
#endif
#endif
