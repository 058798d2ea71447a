// Double-double reference contraction on the device (verification kernel).
//
// R = op(A) * op(B) accumulated in double-double arithmetic: every real
// product x*y is split exactly into p + e (p = fl(x*y), e = fma(x, y, -p),
// TwoProduct) and added to a (hi, lo) pair with Knuth's TwoSum, the error
// terms gathered in lo: the compensated dot product Dot2 of Ogita, Rump and
// Oishi, "Accurate sum and dot product", SIAM J. Sci. Comput. 26(6), 2005.
// Its result is as accurate as a plain dot product computed in twice the
// working precision and then rounded, so R differs from the exact product by
// about 1e-16 of |R| plus 1e-32 of sum |a_l b_l|: at k = 250000 it is a
// reference some 1e17 times tighter than the 1e-14 bar of the FP64 paths.
//
// It is the device counterpart of the CPU Dot2 oracle and exists so that
// results can be checked on the whole C at full problem sizes (a CPU
// double-double GEMM of the 1024 x 1024 x 250000 complex problem takes
// minutes). Inputs of any of the four dtypes are read as double (float
// products are exact in double); R is written as double (complex:
// interleaved), hi and optionally lo parts. Not on any contraction path.
#include <cstdint>

#include "../../../include/splab.h"
#include "common.cuh"

namespace splab {
namespace dd {

constexpr int TM = 32, TN = 32, KT = 32, THREADS = 256;

struct Acc {
  double hi = 0.0, lo = 0.0;
};

// (hi, lo) += x * y, exactly up to the final rounding of lo.
__device__ __forceinline__ void dd_fma(Acc& a, double x, double y) {
  const double p = x * y;
  const double e = fma(x, y, -p);
  const double t = a.hi + p;
  const double z = t - a.hi;
  const double err = (a.hi - (t - z)) + (p - z);
  a.hi = t;
  a.lo += err + e;
}

template <typename S>
__device__ __forceinline__ double2 load_elem(const S* X, int64_t idx, bool cplx, bool conj) {
  if (cplx) {
    const double re = double(X[2 * idx]), im = double(X[2 * idx + 1]);
    return make_double2(re, conj ? -im : im);
  }
  return make_double2(double(X[idx]), 0.0);
}

// One CTA: a 32 x 32 tile of R, 2 x 2 elements per thread; op(A) and op(B)
// tiles of KT along k staged in shared memory (zero outside the problem).
template <typename S, bool CPLX>
__global__ void __launch_bounds__(THREADS)
    dd_gemm_kernel(int opA, int opB, int64_t m, int64_t n, int64_t k, const S* __restrict__ A,
                   int64_t lda, const S* __restrict__ B, int64_t ldb, double* __restrict__ Rhi,
                   double* __restrict__ Rlo, int64_t ldr) {
  __shared__ double2 As[KT][TM + 1];
  __shared__ double2 Bs[KT][TN + 1];
  const int t = threadIdx.x;
  const int tx = t % 16, ty = t / 16;
  const int64_t i0 = int64_t(blockIdx.x) * TM, j0 = int64_t(blockIdx.y) * TN;
  Acc re[2][2], im[2][2];
  for (int64_t l0 = 0; l0 < k; l0 += KT) {
#pragma unroll
    for (int r = 0; r < (KT * TM) / THREADS; ++r) {
      const int e = t + r * THREADS;
      int ii, ll;
      if (opA == 0) {  // op(A)(i, l) = A[i + l lda]: i fastest
        ii = e % TM;
        ll = e / TM;
      } else {  // A[l + i lda]: l fastest
        ll = e % KT;
        ii = e / KT;
      }
      const int64_t gi = i0 + ii, gl = l0 + ll;
      double2 v = make_double2(0.0, 0.0);
      if (gi < m && gl < k)
        v = load_elem(A, opA == 0 ? gi + gl * lda : gl + gi * lda, CPLX, opA == 2);
      As[ll][ii] = v;
    }
#pragma unroll
    for (int r = 0; r < (KT * TN) / THREADS; ++r) {
      const int e = t + r * THREADS;
      int jj, ll;
      if (opB == 0) {  // op(B)(l, j) = B[l + j ldb]: l fastest
        ll = e % KT;
        jj = e / KT;
      } else {  // B[j + l ldb]: j fastest
        jj = e % TN;
        ll = e / TN;
      }
      const int64_t gj = j0 + jj, gl = l0 + ll;
      double2 v = make_double2(0.0, 0.0);
      if (gj < n && gl < k)
        v = load_elem(B, opB == 0 ? gl + gj * ldb : gj + gl * ldb, CPLX, opB == 2);
      Bs[ll][jj] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int l = 0; l < KT; ++l) {
      const double2 a[2] = {As[l][tx], As[l][tx + 16]};
      const double2 b[2] = {Bs[l][ty], Bs[l][ty + 16]};
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int w = 0; w < 2; ++w) {
          dd_fma(re[u][w], a[u].x, b[w].x);
          if (CPLX) {
            dd_fma(re[u][w], -a[u].y, b[w].y);
            dd_fma(im[u][w], a[u].x, b[w].y);
            dd_fma(im[u][w], a[u].y, b[w].x);
          }
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const int64_t gi = i0 + tx + 16 * u, gj = j0 + ty + 16 * w;
      if (gi >= m || gj >= n) continue;
      const Acc* parts[2] = {&re[u][w], &im[u][w]};
      for (int c = 0; c < (CPLX ? 2 : 1); ++c) {
        const double h = parts[c]->hi + parts[c]->lo;
        const double lo = parts[c]->lo - (h - parts[c]->hi);
        const int64_t o = CPLX ? 2 * (gi + gj * ldr) + c : gi + gj * ldr;
        Rhi[o] = h;
        if (Rlo) Rlo[o] = lo;
      }
    }
}

template <typename S, bool CPLX>
cudaError_t launch(int opA, int opB, int64_t m, int64_t n, int64_t k, const void* A, int64_t lda,
                   const void* B, int64_t ldb, double* Rhi, double* Rlo, int64_t ldr,
                   cudaStream_t st) {
  const dim3 grid(unsigned((m + TM - 1) / TM), unsigned((n + TN - 1) / TN));
  dd_gemm_kernel<S, CPLX><<<grid, THREADS, 0, st>>>(opA, opB, m, n, k,
                                                    static_cast<const S*>(A), lda,
                                                    static_cast<const S*>(B), ldb, Rhi, Rlo, ldr);
  return cudaGetLastError();
}

}  // namespace dd
}  // namespace splab

extern "C" SPLAB_API int splab_gemm_dd(int dtype, int opA, int opB, int64_t m, int64_t n,
                                       int64_t k, const void* A, int64_t lda, const void* B,
                                       int64_t ldb, double* Rhi, double* Rlo, int64_t ldr,
                                       void* stream) {
  using namespace splab;
  if (dtype < 0 || dtype > 3 || opA < 0 || opA > 2 || opB < 0 || opB > 2) return SPLAB_ERR_INVALID;
  if (m < 0 || n < 0 || k < 0) return SPLAB_ERR_INVALID;
  if (lda < (opA == 0 ? m : k) || lda < 1 || ldb < (opB == 0 ? k : n) || ldb < 1 ||
      ldr < m || ldr < 1)
    return SPLAB_ERR_INVALID;
  if ((m + dd::TM - 1) / dd::TM > 0x7FFFFFFF || (n + dd::TN - 1) / dd::TN > 65535)
    return SPLAB_ERR_INVALID;
  if (m == 0 || n == 0) return SPLAB_OK;
  if (Rhi == nullptr || (k > 0 && (A == nullptr || B == nullptr))) return SPLAB_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  switch (dtype) {
    case kR32: e = dd::launch<float, false>(opA, opB, m, n, k, A, lda, B, ldb, Rhi, Rlo, ldr, st); break;
    case kR64: e = dd::launch<double, false>(opA, opB, m, n, k, A, lda, B, ldb, Rhi, Rlo, ldr, st); break;
    case kC32: e = dd::launch<float, true>(opA, opB, m, n, k, A, lda, B, ldb, Rhi, Rlo, ldr, st); break;
    default: e = dd::launch<double, true>(opA, opB, m, n, k, A, lda, B, ldb, Rhi, Rlo, ldr, st); break;
  }
  return e == cudaSuccess ? SPLAB_OK : SPLAB_ERR_LAUNCH;
}
