/* C <- alpha * A * B + beta * C for stripe x block -> stripe; reference include/spla/pgemm_sbs.hpp:86-116. Throws the exceptions of spla/exceptions.hpp. */
#ifndef SPLA_PGEMM_SBS_HPP
#define SPLA_PGEMM_SBS_HPP
#include <complex>
#include "spla/config.h"
#include "spla/context.hpp"
#include "spla/matrix_distribution.hpp"
#include "spla/types.h"

namespace spla {
SPLA_EXPORT void pgemm_sbs(int mLocal, int n, int k, float alpha, const float *A, int lda, const float *B,
               int ldb, int bRowOffset, int bColOffset, MatrixDistribution &descB, float beta,
               float *C, int ldc, Context &ctx);

SPLA_EXPORT void pgemm_sbs(int mLocal, int n, int k, double alpha, const double *A, int lda, const double *B,
               int ldb, int bRowOffset, int bColOffset, MatrixDistribution &descB, double beta,
               double *C, int ldc, Context &ctx);

SPLA_EXPORT void pgemm_sbs(int mLocal, int n, int k, std::complex<float> alpha, const std::complex<float> *A, int lda, const std::complex<float> *B,
               int ldb, int bRowOffset, int bColOffset, MatrixDistribution &descB, std::complex<float> beta,
               std::complex<float> *C, int ldc, Context &ctx);

SPLA_EXPORT void pgemm_sbs(int mLocal, int n, int k, std::complex<double> alpha, const std::complex<double> *A, int lda, const std::complex<double> *B,
               int ldb, int bRowOffset, int bColOffset, MatrixDistribution &descB, std::complex<double> beta,
               std::complex<double> *C, int ldc, Context &ctx);

}  // namespace spla
#endif
