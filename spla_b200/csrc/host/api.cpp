// Compute entry points of the SPLA interface: the C++ overloads of
// pgemm_ssb / pgemm_ssbtr / pgemm_sbs / gemm and their spla_* C ABI wrappers.
//
// Validation order and the single-rank shortcut equal the reference's so that
// error codes match:
//   pgemm_ssb(tr): src/pgemm_ssb/pgemm_ssb_host.cpp:157-171 (GPU: pgemm_ssb_gpu.cpp:247-262)
//   pgemm_sbs:     host src/pgemm_sbs/pgemm_sbs_host.cpp:175-183,
//                  GPU  src/pgemm_sbs/pgemm_sbs_gpu.cpp:238-249
//   gemm:          src/gemm/gemm_host.cpp:58-61, src/gemm/gemm_gpu.cpp:63-66
//   parameters:    src/util/check_gemm_param.hpp:36-50
// Deviations (safe supersets): null Context / distribution handles return
// SPLA_INVALID_HANDLE_ERROR; negative B offsets of pgemm_sbs are rejected on the
// host order too (the reference would read out of bounds); distributions over
// more than one rank are rejected with SPLA_MPI_ERROR (the multi-rank ring
// engines are not part of this library).
#include "internal.hpp"
#include "spla/gemm.h"
#include "spla/gemm.hpp"
#include "spla/pgemm_sbs.h"
#include "spla/pgemm_sbs.hpp"
#include "spla/pgemm_ssb.h"
#include "spla/pgemm_ssb.hpp"
#include "spla/pgemm_ssbtr.h"
#include "spla/pgemm_ssbtr.hpp"

namespace spla {
namespace {

void check_gemm_param(SplaOperation opA, SplaOperation opB, long m, long n, long k,
                      const void* A, long lda, const void* B, long ldb, const void* C) {
  if (m < 0 || n < 0 || k < 0) throw InvalidParameterError();
  if ((opA == SPLA_OP_NONE && lda < m) || (opA != SPLA_OP_NONE && lda < k))
    throw InvalidParameterError();
  if ((opB == SPLA_OP_NONE && ldb < k) || (opB != SPLA_OP_NONE && ldb < n))
    throw InvalidParameterError();
  if (k != 0 && m != 0 && !A) throw InvalidPointerError();
  if (k != 0 && n != 0 && !B) throw InvalidPointerError();
  if (n != 0 && m != 0 && !C) throw InvalidPointerError();
}

bool valid_op(SplaOperation op) {
  return op == SPLA_OP_NONE || op == SPLA_OP_TRANSPOSE || op == SPLA_OP_CONJ_TRANSPOSE;
}

template <typename T>
void gemm_impl(SplaOperation opA, SplaOperation opB, int m, int n, int k, T alpha, const T* A,
               int lda, const T* B, int ldb, T beta, T* C, int ldc, ContextInternal& ctx) {
  if (m == 0 || n == 0) return;
  if (!valid_op(opA) || !valid_op(opB)) throw InvalidParameterError();
  check_gemm_param(opA, opB, m, n, k, A, lda, B, ldb, C);
  local_gemm<T>(ctx, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

template <typename T>
void ssb_impl(int m, int n, int kLocal, SplaOperation opA, T alpha, const T* A, int lda,
              const T* B, int ldb, T beta, T* C, int ldc, int cRowOffset, int cColOffset,
              SplaFillMode fill, MatrixDistributionInternal& distC, ContextInternal& ctx) {
  if (m == 0 || n == 0) return;
  if (opA != SPLA_OP_TRANSPOSE && opA != SPLA_OP_CONJ_TRANSPOSE) throw InvalidParameterError();
  if (m < 0 || n < 0 || cRowOffset < 0 || cColOffset < 0) throw InvalidParameterError();
  if (fill != SPLA_FILL_MODE_FULL && fill != SPLA_FILL_MODE_UPPER && fill != SPLA_FILL_MODE_LOWER)
    throw InvalidParameterError();
  if (distC.comm_size() != 1) throw MPIError();
  T* c0 = C ? C + cRowOffset + static_cast<long>(cColOffset) * ldc : C;
  check_gemm_param(opA, SPLA_OP_NONE, m, n, kLocal, A, lda, B, ldb, c0);
  local_gemm<T>(ctx, opA, SPLA_OP_NONE, m, n, kLocal, alpha, A, lda, B, ldb, beta, c0, ldc, fill,
                cRowOffset, cColOffset);
}

template <typename T>
void sbs_impl(int mLocal, int n, int k, T alpha, const T* A, int lda, const T* B, int ldb,
              int bRowOffset, int bColOffset, MatrixDistributionInternal& distB, T beta, T* C,
              int ldc, ContextInternal& ctx) {
  if (k == 0 || n == 0) return;
  if (n < 0 || k < 0 || bRowOffset < 0 || bColOffset < 0) throw InvalidParameterError();
  if (distB.comm_size() != 1 && distB.type() != SPLA_DIST_MIRROR) throw MPIError();
  const T* b0 = B ? B + bRowOffset + static_cast<long>(bColOffset) * ldb : B;
  if (mLocal == 0) return;
  check_gemm_param(SPLA_OP_NONE, SPLA_OP_NONE, mLocal, n, k, A, lda, b0, ldb, C);
  local_gemm<T>(ctx, SPLA_OP_NONE, SPLA_OP_NONE, mLocal, n, k, alpha, A, lda, b0, ldb, beta, C,
                ldc);
}

}  // namespace

#define SPLA_B200_OVERLOADS(T)                                                                    \
  void pgemm_ssbtr(int m, int n, int kLocal, SplaOperation opA, T alpha, const T* A, int lda,     \
                   const T* B, int ldb, T beta, T* C, int ldc, int cRowOffset, int cColOffset,   \
                   SplaFillMode cFillMode, MatrixDistribution& distC, Context& ctx) {            \
    ssb_impl<T>(m, n, kLocal, opA, alpha, A, lda, B, ldb, beta, C, ldc, cRowOffset, cColOffset,  \
                cFillMode, detail::Access::dist(distC), detail::Access::ctx(ctx));               \
  }                                                                                              \
  void pgemm_ssb(int m, int n, int kLocal, SplaOperation opA, T alpha, const T* A, int lda,       \
                 const T* B, int ldb, T beta, T* C, int ldc, int cRowOffset, int cColOffset,     \
                 MatrixDistribution& distC, Context& ctx) {                                      \
    ssb_impl<T>(m, n, kLocal, opA, alpha, A, lda, B, ldb, beta, C, ldc, cRowOffset, cColOffset,  \
                SPLA_FILL_MODE_FULL, detail::Access::dist(distC), detail::Access::ctx(ctx));     \
  }                                                                                              \
  void pgemm_sbs(int mLocal, int n, int k, T alpha, const T* A, int lda, const T* B, int ldb,     \
                 int bRowOffset, int bColOffset, MatrixDistribution& descB, T beta, T* C,        \
                 int ldc, Context& ctx) {                                                        \
    sbs_impl<T>(mLocal, n, k, alpha, A, lda, B, ldb, bRowOffset, bColOffset,                     \
                detail::Access::dist(descB), beta, C, ldc, detail::Access::ctx(ctx));            \
  }                                                                                              \
  void gemm(SplaOperation opA, SplaOperation opB, int m, int n, int k, T alpha, const T* A,       \
            int lda, const T* B, int ldb, T beta, T* C, int ldc, Context& ctx) {                 \
    gemm_impl<T>(opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,                         \
                 detail::Access::ctx(ctx));                                                      \
  }

SPLA_B200_OVERLOADS(float)
SPLA_B200_OVERLOADS(double)
SPLA_B200_OVERLOADS(std::complex<float>)
SPLA_B200_OVERLOADS(std::complex<double>)
#undef SPLA_B200_OVERLOADS

}  // namespace spla

// ---------------------------------------------------------------------------
// C ABI (reference src/spla/pgemm_ssb.cpp:78-111, pgemm_ssbtr.cpp:122-195,
// pgemm_sbs.cpp:120-194, gemm.cpp:110-172): exceptions become SplaError codes.

namespace {
template <typename F>
SplaError guarded(F&& f) {
  try {
    f();
  } catch (const spla::GenericError& e) {
    return e.error_code();
  } catch (...) {
    return SPLA_UNKNOWN_ERROR;
  }
  return SPLA_SUCCESS;
}
spla::Context& ctx_of(SplaContext c) { return *static_cast<spla::Context*>(c); }
spla::MatrixDistribution& dist_of(SplaMatrixDistribution d) {
  return *static_cast<spla::MatrixDistribution*>(d);
}
using cf = std::complex<float>;
using cd = std::complex<double>;
template <typename T>
T scalar(const void* p) {
  return *static_cast<const T*>(p);
}
}  // namespace

extern "C" {

#define SPLA_B200_SSBTR_C(NAME, T, AT, PT)                                                        \
  SplaError NAME(int m, int n, int kLocal, SplaOperation opA, AT alpha, const PT* A, int lda,     \
                 const PT* B, int ldb, AT beta, PT* C, int ldc, int cRowOffset, int cColOffset,  \
                 SplaFillMode cFillMode, SplaMatrixDistribution distC, SplaContext ctx) {        \
    if (!ctx || !distC) return SPLA_INVALID_HANDLE_ERROR;                                        \
    return guarded([&] {                                                                         \
      spla::pgemm_ssbtr(m, n, kLocal, opA, scalar<T>(&alpha), static_cast<const T*>(A), lda,    \
                        static_cast<const T*>(B), ldb, scalar<T>(&beta), static_cast<T*>(C),     \
                        ldc, cRowOffset, cColOffset, cFillMode, dist_of(distC), ctx_of(ctx));    \
    });                                                                                          \
  }
#define SPLA_B200_SSB_C(NAME, T, AT, PT)                                                          \
  SplaError NAME(int m, int n, int kLocal, SplaOperation opA, AT alpha, const PT* A, int lda,     \
                 const PT* B, int ldb, AT beta, PT* C, int ldc, int cRowOffset, int cColOffset,  \
                 SplaMatrixDistribution distC, SplaContext ctx) {                                \
    if (!ctx || !distC) return SPLA_INVALID_HANDLE_ERROR;                                        \
    return guarded([&] {                                                                         \
      spla::pgemm_ssb(m, n, kLocal, opA, scalar<T>(&alpha), static_cast<const T*>(A), lda,      \
                      static_cast<const T*>(B), ldb, scalar<T>(&beta), static_cast<T*>(C), ldc,  \
                      cRowOffset, cColOffset, dist_of(distC), ctx_of(ctx));                      \
    });                                                                                          \
  }
#define SPLA_B200_SBS_C(NAME, T, AT, PT)                                                          \
  SplaError NAME(int mLocal, int n, int k, AT alpha, const PT* A, int lda, const PT* B, int ldb,  \
                 int bRowOffset, int bColOffset, SplaMatrixDistribution distB, AT beta, PT* C,   \
                 int ldc, SplaContext ctx) {                                                     \
    if (!ctx || !distB) return SPLA_INVALID_HANDLE_ERROR;                                        \
    return guarded([&] {                                                                         \
      spla::pgemm_sbs(mLocal, n, k, scalar<T>(&alpha), static_cast<const T*>(A), lda,           \
                      static_cast<const T*>(B), ldb, bRowOffset, bColOffset, dist_of(distB),     \
                      scalar<T>(&beta), static_cast<T*>(C), ldc, ctx_of(ctx));                   \
    });                                                                                          \
  }
#define SPLA_B200_GEMM_C(NAME, T, AT, PT)                                                         \
  SplaError NAME(SplaOperation opA, SplaOperation opB, int m, int n, int k, AT alpha,             \
                 const PT* A, int lda, const PT* B, int ldb, AT beta, PT* C, int ldc,            \
                 SplaContext ctx) {                                                              \
    if (!ctx) return SPLA_INVALID_HANDLE_ERROR;                                                  \
    return guarded([&] {                                                                         \
      spla::gemm(opA, opB, m, n, k, scalar<T>(&alpha), static_cast<const T*>(A), lda,           \
                 static_cast<const T*>(B), ldb, scalar<T>(&beta), static_cast<T*>(C), ldc,       \
                 ctx_of(ctx));                                                                   \
    });                                                                                          \
  }

// Real dtypes take alpha/beta by value; complex ones by pointer to (re, im).
// `scalar<T>(&alpha)` reads the value for real types; for complex types the
// macro argument AT is `const void*`, handled by the specialisations below.
SPLA_B200_SSBTR_C(spla_psgemm_ssbtr, float, float, float)
SPLA_B200_SSBTR_C(spla_pdgemm_ssbtr, double, double, double)
SPLA_B200_SSB_C(spla_psgemm_ssb, float, float, float)
SPLA_B200_SSB_C(spla_pdgemm_ssb, double, double, double)
SPLA_B200_SBS_C(spla_psgemm_sbs, float, float, float)
SPLA_B200_SBS_C(spla_pdgemm_sbs, double, double, double)
SPLA_B200_GEMM_C(spla_sgemm, float, float, float)
SPLA_B200_GEMM_C(spla_dgemm, double, double, double)

#undef SPLA_B200_SSBTR_C
#undef SPLA_B200_SSB_C
#undef SPLA_B200_SBS_C
#undef SPLA_B200_GEMM_C

#define SPLA_B200_CPLX_ENTRIES(PFX, T)                                                            \
  SplaError spla_p##PFX##gemm_ssbtr(int m, int n, int kLocal, SplaOperation opA,                  \
                                    const void* alpha, const void* A, int lda, const void* B,    \
                                    int ldb, const void* beta, void* C, int ldc, int cRowOffset, \
                                    int cColOffset, SplaFillMode cFillMode,                      \
                                    SplaMatrixDistribution distC, SplaContext ctx) {             \
    if (!ctx || !distC) return SPLA_INVALID_HANDLE_ERROR;                                        \
    if (!alpha || !beta) return SPLA_INVALID_POINTER_ERROR;                                      \
    return guarded([&] {                                                                         \
      spla::pgemm_ssbtr(m, n, kLocal, opA, scalar<T>(alpha), static_cast<const T*>(A), lda,     \
                        static_cast<const T*>(B), ldb, scalar<T>(beta), static_cast<T*>(C), ldc, \
                        cRowOffset, cColOffset, cFillMode, dist_of(distC), ctx_of(ctx));         \
    });                                                                                          \
  }                                                                                              \
  SplaError spla_p##PFX##gemm_ssb(int m, int n, int kLocal, SplaOperation opA, const void* alpha, \
                                  const void* A, int lda, const void* B, int ldb,                \
                                  const void* beta, void* C, int ldc, int cRowOffset,            \
                                  int cColOffset, SplaMatrixDistribution distC, SplaContext ctx) { \
    if (!ctx || !distC) return SPLA_INVALID_HANDLE_ERROR;                                        \
    if (!alpha || !beta) return SPLA_INVALID_POINTER_ERROR;                                      \
    return guarded([&] {                                                                         \
      spla::pgemm_ssb(m, n, kLocal, opA, scalar<T>(alpha), static_cast<const T*>(A), lda,       \
                      static_cast<const T*>(B), ldb, scalar<T>(beta), static_cast<T*>(C), ldc,   \
                      cRowOffset, cColOffset, dist_of(distC), ctx_of(ctx));                      \
    });                                                                                          \
  }                                                                                              \
  SplaError spla_p##PFX##gemm_sbs(int mLocal, int n, int k, const void* alpha, const void* A,     \
                                  int lda, const void* B, int ldb, int bRowOffset,               \
                                  int bColOffset, SplaMatrixDistribution distB, const void* beta, \
                                  void* C, int ldc, SplaContext ctx) {                           \
    if (!ctx || !distB) return SPLA_INVALID_HANDLE_ERROR;                                        \
    if (!alpha || !beta) return SPLA_INVALID_POINTER_ERROR;                                      \
    return guarded([&] {                                                                         \
      spla::pgemm_sbs(mLocal, n, k, scalar<T>(alpha), static_cast<const T*>(A), lda,            \
                      static_cast<const T*>(B), ldb, bRowOffset, bColOffset, dist_of(distB),     \
                      scalar<T>(beta), static_cast<T*>(C), ldc, ctx_of(ctx));                    \
    });                                                                                          \
  }                                                                                              \
  SplaError spla_##PFX##gemm(SplaOperation opA, SplaOperation opB, int m, int n, int k,           \
                             const void* alpha, const void* A, int lda, const void* B, int ldb,  \
                             const void* beta, void* C, int ldc, SplaContext ctx) {              \
    if (!ctx) return SPLA_INVALID_HANDLE_ERROR;                                                  \
    if (!alpha || !beta) return SPLA_INVALID_POINTER_ERROR;                                      \
    return guarded([&] {                                                                         \
      spla::gemm(opA, opB, m, n, k, scalar<T>(alpha), static_cast<const T*>(A), lda,            \
                 static_cast<const T*>(B), ldb, scalar<T>(beta), static_cast<T*>(C), ldc,        \
                 ctx_of(ctx));                                                                   \
    });                                                                                          \
  }

SPLA_B200_CPLX_ENTRIES(c, cf)
SPLA_B200_CPLX_ENTRIES(z, cd)
#undef SPLA_B200_CPLX_ENTRIES

}  // extern "C"
