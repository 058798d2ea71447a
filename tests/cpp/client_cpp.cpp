// A C++ application written against the reference's C++ interface, compiled
// against include/ and linked with libspla.so: spla::Context,
// spla::MatrixDistribution, spla::pgemm_ssb (complex float, host vectors: the
// k-streamed path), spla::pgemm_ssbtr (double, upper fill, C offsets) and spla::gemm (all op
// pairs for complex double), each checked against a long-double loop, and the
// exception mapping of an invalid call. Prints "OK" and exits 0 on success.
#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

#include <spla/spla.hpp>
#include <spla/pgemm_ssbtr.hpp>

using cd = std::complex<double>;
using cf = std::complex<float>;

static int fail(const char* what, double err) {
  std::printf("FAIL %s %.3e\n", what, err);
  return 1;
}

template <typename T>
static T op_elem(const std::vector<T>& X, int ld, int r, int c, SplaOperation op) {
  // element (r, c) of op(X), X column-major with leading dimension ld
  if (op == SPLA_OP_NONE) return X[r + static_cast<long>(c) * ld];
  const T v = X[c + static_cast<long>(r) * ld];
  if constexpr (std::is_same_v<T, cd>) return op == SPLA_OP_CONJ_TRANSPOSE ? std::conj(v) : v;
  return v;
}

int main() {
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  try {
    spla::Context ctx(SPLA_PU_GPU);
    auto dist = spla::MatrixDistribution::create_blacs_block_cyclic(MPI_COMM_SELF, 'R', 1, 1, 64,
                                                                     64);
    {  // complex float ssb
      const int m = 40, n = 33, k = 50000;
      std::vector<cf> A(static_cast<size_t>(k) * m), B(static_cast<size_t>(k) * n), C(m * n);
      for (auto& x : A) x = cf(float(u(rng)), float(u(rng)));
      for (auto& x : B) x = cf(float(u(rng)), float(u(rng)));
      spla::pgemm_ssb(m, n, k, SPLA_OP_CONJ_TRANSPOSE, cf(1.f), A.data(), k, B.data(), k, cf(0.f),
                      C.data(), m, 0, 0, dist, ctx);
      double num = 0, den = 0;
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
          long double re = 0, im = 0;
          for (int l = 0; l < k; ++l) {
            const cd a = std::conj(cd(A[static_cast<size_t>(i) * k + l]));
            const cd b = cd(B[static_cast<size_t>(j) * k + l]);
            re += (long double)a.real() * b.real() - (long double)a.imag() * b.imag();
            im += (long double)a.real() * b.imag() + (long double)a.imag() * b.real();
          }
          const cd d = cd(C[i + j * m]) - cd(double(re), double(im));
          num += std::norm(d);
          den += double(re * re + im * im);
        }
      if (!(std::sqrt(num / den) <= 1e-6)) return fail("pgemm_ssb cf", std::sqrt(num / den));
    }
    {  // double ssbtr, upper fill, C block at offset (3, 5) inside a padded C
      const int m = 70, n = 60, k = 9000, ro = 3, co = 5, ldc = m + ro + 4;
      std::vector<double> A(static_cast<size_t>(k) * m), B(static_cast<size_t>(k) * n);
      std::vector<double> C(static_cast<size_t>(ldc) * (n + co)), C0;
      for (auto& x : A) x = u(rng);
      for (auto& x : B) x = u(rng);
      for (auto& x : C) x = u(rng);
      C0 = C;
      spla::pgemm_ssbtr(m, n, k, SPLA_OP_TRANSPOSE, 1.5, A.data(), k, B.data(), k, -0.5, C.data(),
                        ldc, ro, co, SPLA_FILL_MODE_UPPER, dist, ctx);
      double num = 0, den = 0;
      for (int j = 0; j < n; ++j)
        for (int i = 0; i <= j && i < m; ++i) {  // the requested triangle of the block
          long double s = 0;
          for (int l = 0; l < k; ++l)
            s += (long double)A[static_cast<size_t>(i) * k + l] * B[static_cast<size_t>(j) * k + l];
          const long idx = (i + ro) + static_cast<long>(j + co) * ldc;
          const long double want = 1.5L * s - 0.5L * C0[idx];
          num += std::pow(C[idx] - double(want), 2);
          den += double(want * want);
        }
      if (!(std::sqrt(num / den) <= 1e-14)) return fail("pgemm_ssbtr d", std::sqrt(num / den));
      for (int j = 0; j < n + co; ++j)  // outside the block: untouched
        for (int i = 0; i < ldc; ++i) {
          const bool inside = i >= ro && i < ro + m && j >= co;
          if (!inside && C[i + static_cast<long>(j) * ldc] != C0[i + static_cast<long>(j) * ldc])
            return fail("pgemm_ssbtr outside block", 0);
        }
    }
    {  // gemm, complex double, all nine op pairs
      const int m = 21, n = 17, k = 33;
      const SplaOperation ops[3] = {SPLA_OP_NONE, SPLA_OP_TRANSPOSE, SPLA_OP_CONJ_TRANSPOSE};
      for (SplaOperation oa : ops)
        for (SplaOperation ob : ops) {
          const int lda = (oa == SPLA_OP_NONE ? m : k) + 2, ldb = (ob == SPLA_OP_NONE ? k : n) + 3;
          std::vector<cd> A(static_cast<size_t>(lda) * (oa == SPLA_OP_NONE ? k : m));
          std::vector<cd> B(static_cast<size_t>(ldb) * (ob == SPLA_OP_NONE ? n : k));
          std::vector<cd> C(m * n);
          for (auto& x : A) x = cd(u(rng), u(rng));
          for (auto& x : B) x = cd(u(rng), u(rng));
          for (auto& x : C) x = cd(u(rng), u(rng));
          const std::vector<cd> C0 = C;
          const cd alpha(0.5, -1.0), beta(0.25, 0.5);
          spla::gemm(oa, ob, m, n, k, alpha, A.data(), lda, B.data(), ldb, beta, C.data(), m, ctx);
          double num = 0, den = 0;
          for (int j = 0; j < n; ++j)
            for (int i = 0; i < m; ++i) {
              cd s = 0;
              for (int l = 0; l < k; ++l) s += op_elem(A, lda, i, l, oa) * op_elem(B, ldb, l, j, ob);
              const cd want = alpha * s + beta * C0[i + j * m];
              num += std::norm(C[i + j * m] - want);
              den += std::norm(want);
            }
          if (!(std::sqrt(num / den) <= 1e-13)) return fail("gemm z", std::sqrt(num / den));
        }
    }
    bool thrown = false;  // lda < k is rejected like the reference (check_gemm_param)
    try {
      std::vector<double> A(100), B(100), C(100);
      spla::pgemm_ssb(4, 4, 10, SPLA_OP_TRANSPOSE, 1.0, A.data(), 5, B.data(), 10, 0.0, C.data(), 4,
                      0, 0, dist, ctx);
    } catch (const spla::InvalidParameterError&) {
      thrown = true;
    }
    if (!thrown) return fail("invalid lda not rejected", 0);
  } catch (const spla::GenericError& e) {
    std::printf("FAIL exception %s\n", e.what());
    return 1;
  }
  std::printf("OK\n");
  return 0;
}
