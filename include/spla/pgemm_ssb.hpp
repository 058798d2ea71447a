/* C <- alpha * op(A) * B + beta * C for stripe x stripe -> block; reference include/spla/pgemm_ssb.hpp:88-117. Throws the exceptions of spla/exceptions.hpp. */
#ifndef SPLA_PGEMM_SSB_HPP
#define SPLA_PGEMM_SSB_HPP
#include <complex>
#include "spla/config.h"
#include "spla/context.hpp"
#include "spla/matrix_distribution.hpp"
#include "spla/types.h"

namespace spla {
SPLA_EXPORT void pgemm_ssb(int m, int n, int kLocal, SplaOperation opA, float alpha, const float *A, int lda,
               const float *B, int ldb, float beta, float *C, int ldc, int cRowOffset,
               int cColOffset, MatrixDistribution &distC, Context &ctx);

SPLA_EXPORT void pgemm_ssb(int m, int n, int kLocal, SplaOperation opA, double alpha, const double *A, int lda,
               const double *B, int ldb, double beta, double *C, int ldc, int cRowOffset,
               int cColOffset, MatrixDistribution &distC, Context &ctx);

SPLA_EXPORT void pgemm_ssb(int m, int n, int kLocal, SplaOperation opA, std::complex<float> alpha, const std::complex<float> *A, int lda,
               const std::complex<float> *B, int ldb, std::complex<float> beta, std::complex<float> *C, int ldc, int cRowOffset,
               int cColOffset, MatrixDistribution &distC, Context &ctx);

SPLA_EXPORT void pgemm_ssb(int m, int n, int kLocal, SplaOperation opA, std::complex<double> alpha, const std::complex<double> *A, int lda,
               const std::complex<double> *B, int ldb, std::complex<double> beta, std::complex<double> *C, int ldc, int cRowOffset,
               int cColOffset, MatrixDistribution &distC, Context &ctx);

}  // namespace spla
#endif
