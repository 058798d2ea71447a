/* A C application written against the reference's C interface, compiled
 * against include/ and linked with libspla.so: complex double pgemm_ssb
 * (C = A^H B, host operands, so the k-streamed path runs), float pgemm_ssbtr
 * (lower fill) and double pgemm_sbs, each checked against a long-double loop.
 * Prints "OK" and exits 0 on success. */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <spla/spla.h>
#include <spla/pgemm_ssbtr.h>

static unsigned long long state = 88172645463325252ull;
static double uni(void) { /* xorshift64, uniform in [-1, 1) */
  state ^= state << 13;
  state ^= state >> 7;
  state ^= state << 17;
  return (double)(state >> 11) / 4503599627370496.0 - 1.0;
}

static int fail(const char *what, double err) {
  printf("FAIL %s %.3e\n", what, err);
  return 1;
}

int main(void) {
  SplaContext ctx;
  if (spla_ctx_create(&ctx, SPLA_PU_GPU) != SPLA_SUCCESS) return fail("ctx", 0);
  SplaMatrixDistribution dist;
  if (spla_mat_dis_create_block_cyclic(&dist, MPI_COMM_SELF, 'R', 1, 1, 64, 64) != SPLA_SUCCESS)
    return fail("dist", 0);

  /* complex double ssb */
  {
    const int m = 37, n = 29, k = 70000;
    double complex *A = malloc(sizeof(double complex) * k * m);
    double complex *B = malloc(sizeof(double complex) * k * n);
    double complex *C = malloc(sizeof(double complex) * m * n);
    for (long i = 0; i < (long)k * m; ++i) A[i] = uni() + I * uni();
    for (long i = 0; i < (long)k * n; ++i) B[i] = uni() + I * uni();
    double complex alpha = 1.0, beta = 0.0;
    if (spla_pzgemm_ssb(m, n, k, SPLA_OP_CONJ_TRANSPOSE, &alpha, A, k, B, k, &beta, C, m, 0, 0,
                        dist, ctx) != SPLA_SUCCESS)
      return fail("pzgemm_ssb", 0);
    double num = 0, den = 0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) {
        long double re = 0, im = 0;
        for (int l = 0; l < k; ++l) {
          const double complex a = conj(A[(long)i * k + l]), b = B[(long)j * k + l];
          re += (long double)creal(a) * creal(b) - (long double)cimag(a) * cimag(b);
          im += (long double)creal(a) * cimag(b) + (long double)cimag(a) * creal(b);
        }
        const double complex d = C[i + (long)j * m] - ((double)re + I * (double)im);
        num += creal(d) * creal(d) + cimag(d) * cimag(d);
        den += (double)(re * re + im * im);
      }
    if (!(sqrt(num / den) <= 1e-14)) return fail("pzgemm_ssb error", sqrt(num / den));
    free(A);
    free(B);
    free(C);
  }

  /* float ssbtr, lower triangle */
  {
    const int m = 50, n = 50, k = 30000;
    float *A = malloc(sizeof(float) * k * m), *B = malloc(sizeof(float) * k * n);
    float *C = malloc(sizeof(float) * m * n);
    for (long i = 0; i < (long)k * m; ++i) A[i] = (float)uni();
    for (long i = 0; i < (long)k * n; ++i) B[i] = (float)uni();
    for (int i = 0; i < m * n; ++i) C[i] = 0.f;
    if (spla_psgemm_ssbtr(m, n, k, SPLA_OP_TRANSPOSE, 1.f, A, k, B, k, 0.f, C, m, 0, 0,
                          SPLA_FILL_MODE_LOWER, dist, ctx) != SPLA_SUCCESS)
      return fail("psgemm_ssbtr", 0);
    double num = 0, den = 0;
    for (int j = 0; j < n; ++j)
      for (int i = j; i < m; ++i) {
        long double s = 0;
        for (int l = 0; l < k; ++l) s += (long double)A[(long)i * k + l] * B[(long)j * k + l];
        const double d = C[i + j * m] - (double)s;
        num += d * d;
        den += (double)(s * s);
      }
    if (!(sqrt(num / den) <= 1e-6)) return fail("psgemm_ssbtr error", sqrt(num / den));
    free(A);
    free(B);
    free(C);
  }

  /* double sbs: C (mLocal x n) = alpha A (mLocal x k) B (k x n block) + beta C */
  {
    const int ml = 300, n = 40, k = 40;
    double *A = malloc(sizeof(double) * ml * k), *B = malloc(sizeof(double) * k * n);
    double *C = malloc(sizeof(double) * ml * n), *C0 = malloc(sizeof(double) * ml * n);
    for (int i = 0; i < ml * k; ++i) A[i] = uni();
    for (int i = 0; i < k * n; ++i) B[i] = uni();
    for (int i = 0; i < ml * n; ++i) C0[i] = C[i] = uni();
    if (spla_pdgemm_sbs(ml, n, k, 2.0, A, ml, B, k, 0, 0, dist, 0.5, C, ml, ctx) != SPLA_SUCCESS)
      return fail("pdgemm_sbs", 0);
    double num = 0, den = 0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < ml; ++i) {
        long double s = 0;
        for (int l = 0; l < k; ++l) s += (long double)A[i + l * ml] * B[l + j * k];
        const long double want = 2.0L * s + 0.5L * C0[i + j * ml];
        const double d = C[i + j * ml] - (double)want;
        num += d * d;
        den += (double)(want * want);
      }
    if (!(sqrt(num / den) <= 1e-14)) return fail("pdgemm_sbs error", sqrt(num / den));
    free(A);
    free(B);
    free(C);
    free(C0);
  }

  spla_mat_dis_destroy(&dist);
  spla_ctx_destroy(&ctx);
  printf("OK\n");
  return 0;
}
