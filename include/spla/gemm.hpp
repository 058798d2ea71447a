/* local C <- alpha * op(A) * op(B) + beta * C; reference include/spla/gemm.hpp:66-97. Throws the exceptions of spla/exceptions.hpp. */
#ifndef SPLA_GEMM_HPP
#define SPLA_GEMM_HPP
#include <complex>
#include "spla/config.h"
#include "spla/context.hpp"
#include "spla/matrix_distribution.hpp"
#include "spla/types.h"

namespace spla {
SPLA_EXPORT void gemm(SplaOperation opA, SplaOperation opB, int m, int n, int k, float alpha, const float *A,
          int lda, const float *B, int ldb, float beta, float *C, int ldc, Context &ctx);

SPLA_EXPORT void gemm(SplaOperation opA, SplaOperation opB, int m, int n, int k, double alpha, const double *A,
          int lda, const double *B, int ldb, double beta, double *C, int ldc, Context &ctx);

SPLA_EXPORT void gemm(SplaOperation opA, SplaOperation opB, int m, int n, int k, std::complex<float> alpha, const std::complex<float> *A,
          int lda, const std::complex<float> *B, int ldb, std::complex<float> beta, std::complex<float> *C, int ldc, Context &ctx);

SPLA_EXPORT void gemm(SplaOperation opA, SplaOperation opB, int m, int n, int k, std::complex<double> alpha, const std::complex<double> *A,
          int lda, const std::complex<double> *B, int ldb, std::complex<double> beta, std::complex<double> *C, int ldc, Context &ctx);

}  // namespace spla
#endif
