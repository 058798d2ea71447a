/*
 * ORACLE — test infrastructure only. Nothing in the product links, loads or
 * calls this file; only tests/, the smoke check and bench.py's CPU-baseline
 * leg do, and only as the checker.
 *
 * A plain-C restatement of the single-rank SPLA local contraction path with a
 * compensated (double-double) accumulator, so that it can serve as the
 * accuracy reference ("FP64 oracle") the GPU kernels are measured against:
 *
 *   - oracle_check_gemm_param  follows src/util/check_gemm_param.hpp:36-50
 *   - oracle_gemm              follows src/gemm/gemm_host.cpp:55-72 (early exit,
 *                              validation, ld clamp) with C = a*op(A)*op(B) + b*C
 *                              evaluated as in src/util/blas_interface.cpp:103-192
 *                              but in double-double arithmetic
 *   - oracle_pgemm_ssb         follows src/pgemm_ssb/pgemm_ssb_host.cpp:151-171
 *                              (validation order, single-rank shortcut, C offset)
 *   - oracle_pgemm_sbs         follows src/pgemm_sbs/pgemm_sbs_host.cpp:171-183 (host
 *                              order) and src/pgemm_sbs/pgemm_sbs_gpu.cpp:234-249
 *                              (GPU order) selected by `gpu_order`
 *   - oracle_block_info        follows src/block_generation/block_cyclic_generator.cpp:59-100
 *   - oracle_block_is_active   follows src/block_generation/block.hpp:58-66
 *   - oracle_local_size        follows src/block_generation/block_cyclic_generator.cpp:117-141
 *
 * Dot products use Ogita, Rump & Oishi, "Accurate sum and dot product",
 * SIAM J. Sci. Comput. 26(6), 2005 (algorithm Dot2: TwoProduct via fma,
 * TwoSum), which is as accurate as evaluating in twice the working precision.
 *
 * dtype codes: 0 = float, 1 = double, 2 = complex float, 3 = complex double
 * (interleaved re,im). op codes follow SplaOperation: 0 = N, 1 = T, 2 = C.
 * Return codes follow SplaError: 0 success, 3 invalid parameter, 4 invalid pointer.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#define OR_SUCCESS 0
#define OR_INVALID_PARAMETER 3
#define OR_INVALID_POINTER 4

typedef struct {
  double hi, lo;
} dd_t;

static inline void two_sum(double a, double b, double *s, double *e) {
  double x = a + b;
  double z = x - a;
  *e = (a - (x - z)) + (b - z);
  *s = x;
}

/* Dot2 accumulator: p carries the running sum, s the accumulated errors. */
typedef struct {
  double p, s;
} dot2_t;

static inline void dot2_add(dot2_t *acc, double x, double y) {
  double h = x * y;
  double r = fma(x, y, -h);
  double q;
  two_sum(acc->p, h, &acc->p, &q);
  acc->s += q + r;
}

static inline dd_t dot2_result(const dot2_t *acc) {
  dd_t out;
  two_sum(acc->p, acc->s, &out.hi, &out.lo);
  return out;
}

/* check_gemm_param (src/util/check_gemm_param.hpp:36-50) */
int oracle_check_gemm_param(int opA, int opB, long m, long n, long k, const void *A, long lda,
                            const void *B, long ldb, const void *C, long ldc) {
  (void)ldc;
  if (m < 0 || n < 0 || k < 0) return OR_INVALID_PARAMETER;
  if ((opA == 0 && lda < m) || (opA != 0 && lda < k)) return OR_INVALID_PARAMETER;
  if ((opB == 0 && ldb < k) || (opB != 0 && ldb < n)) return OR_INVALID_PARAMETER;
  if ((k != 0 && m != 0) && !A) return OR_INVALID_POINTER;
  if ((k != 0 && n != 0) && !B) return OR_INVALID_POINTER;
  if ((n != 0 && m != 0) && !C) return OR_INVALID_POINTER;
  return OR_SUCCESS;
}

/* element (row i, col l) of op(A) where op(A) is m x k; returns re/im in double */
static inline void load_op(int cplx, int isdouble, int op, const void *X, long ld, long i, long l,
                           double *re, double *im) {
  long idx = (op == 0) ? (i + l * ld) : (l + i * ld);
  if (cplx) {
    if (isdouble) {
      const double *p = (const double *)X + 2 * idx;
      *re = p[0];
      *im = p[1];
    } else {
      const float *p = (const float *)X + 2 * idx;
      *re = p[0];
      *im = p[1];
    }
    if (op == 2) *im = -*im;
  } else {
    *re = isdouble ? ((const double *)X)[idx] : (double)((const float *)X)[idx];
    *im = 0.0;
  }
}

/*
 * C(m x n) = alpha * op(A)(m x k) * op(B)(k x n) + beta * C, column major,
 * each element's dot product accumulated with Dot2, then alpha/beta applied
 * with one more compensated step. If C_lo is non-null, the low part of the
 * double-double result (before alpha/beta, only meaningful for alpha=1,
 * beta=0) is written there with the same layout as C (real: ldc doubles,
 * complex: 2*ldc doubles); C_lo is always double precision.
 */
int oracle_gemm(int dtype, int opA, int opB, long m, long n, long k, const void *alpha,
                const void *A, long lda, const void *B, long ldb, const void *beta, void *C,
                long ldc, double *C_lo) {
  if (m == 0 || n == 0) return OR_SUCCESS;
  int rc = oracle_check_gemm_param(opA, opB, m, n, k, A, lda, B, ldb, C, ldc);
  if (rc) return rc;
  if (lda < 1) lda = 1;
  if (ldb < 1) ldb = 1;
  if (ldc < 1) ldc = 1;
  const int cplx = dtype >= 2;
  const int isdouble = (dtype == 1 || dtype == 3);
  double ar, ai, br, bi;
  if (isdouble) {
    ar = ((const double *)alpha)[0];
    ai = cplx ? ((const double *)alpha)[1] : 0.0;
    br = ((const double *)beta)[0];
    bi = cplx ? ((const double *)beta)[1] : 0.0;
  } else {
    ar = ((const float *)alpha)[0];
    ai = cplx ? ((const float *)alpha)[1] : 0.0;
    br = ((const float *)beta)[0];
    bi = cplx ? ((const float *)beta)[1] : 0.0;
  }

#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (long j = 0; j < n; ++j) {
    for (long i = 0; i < m; ++i) {
      dot2_t re = {0.0, 0.0}, im = {0.0, 0.0};
      for (long l = 0; l < k; ++l) {
        double xr, xi, yr, yi;
        load_op(cplx, isdouble, opA, A, lda, i, l, &xr, &xi);
        /* op(B) is k x n: element (l, j); B itself is k x n for N, n x k otherwise */
        load_op(cplx, isdouble, opB == 0 ? 1 : 0, B, ldb, j, l, &yr, &yi);
        if (opB == 2) yi = -yi;
        dot2_add(&re, xr, yr);
        if (cplx) {
          dot2_add(&re, -xi, yi);
          dot2_add(&im, xr, yi);
          dot2_add(&im, xi, yr);
        }
      }
      dd_t dr = dot2_result(&re);
      dd_t di = dot2_result(&im);
      long cidx = i + j * ldc;
      double cr = 0.0, ci = 0.0;
      if (br != 0.0 || bi != 0.0) {
        if (isdouble) {
          cr = ((double *)C)[cplx ? 2 * cidx : cidx];
          ci = cplx ? ((double *)C)[2 * cidx + 1] : 0.0;
        } else {
          cr = ((float *)C)[cplx ? 2 * cidx : cidx];
          ci = cplx ? ((float *)C)[2 * cidx + 1] : 0.0;
        }
      }
      /* alpha*(d) + beta*c, accumulated with Dot2 over the hi and lo parts */
      dot2_t outr = {0.0, 0.0}, outi = {0.0, 0.0};
      dot2_add(&outr, ar, dr.hi);
      dot2_add(&outr, ar, dr.lo);
      dot2_add(&outr, -ai, di.hi);
      dot2_add(&outr, -ai, di.lo);
      dot2_add(&outr, br, cr);
      dot2_add(&outr, -bi, ci);
      dot2_add(&outi, ar, di.hi);
      dot2_add(&outi, ar, di.lo);
      dot2_add(&outi, ai, dr.hi);
      dot2_add(&outi, ai, dr.lo);
      dot2_add(&outi, br, ci);
      dot2_add(&outi, bi, cr);
      dd_t fr = dot2_result(&outr);
      dd_t fi = dot2_result(&outi);
      if (isdouble) {
        if (cplx) {
          ((double *)C)[2 * cidx] = fr.hi;
          ((double *)C)[2 * cidx + 1] = fi.hi;
        } else {
          ((double *)C)[cidx] = fr.hi;
        }
      } else {
        /* round the double-double to float: hi+lo rounded once */
        if (cplx) {
          ((float *)C)[2 * cidx] = (float)(fr.hi + fr.lo);
          ((float *)C)[2 * cidx + 1] = (float)(fi.hi + fi.lo);
        } else {
          ((float *)C)[cidx] = (float)(fr.hi + fr.lo);
        }
      }
      if (C_lo) {
        if (cplx) {
          C_lo[2 * cidx] = fr.lo;
          C_lo[2 * cidx + 1] = fi.lo;
        } else {
          C_lo[cidx] = fr.lo;
        }
      }
    }
  }
  return OR_SUCCESS;
}

static size_t elem_size(int dtype) {
  switch (dtype) {
    case 0: return 4;
    case 1: return 8;
    case 2: return 8;
    default: return 16;
  }
}

/*
 * Single-rank pgemm_ssb / pgemm_ssbtr: src/pgemm_ssb/pgemm_ssb_host.cpp:157-171
 * (the GPU entry src/pgemm_ssb/pgemm_ssb_gpu.cpp:247-262 has the same order).
 * On one rank the fill mode is not used: the full C block is computed.
 */
int oracle_pgemm_ssb(int dtype, int m, int n, int kLocal, int opA, const void *alpha,
                     const void *A, int lda, const void *B, int ldb, const void *beta, void *C,
                     int ldc, int cRowOffset, int cColOffset) {
  if (m == 0 || n == 0) return OR_SUCCESS;
  if (opA != 1 && opA != 2) return OR_INVALID_PARAMETER;
  if (m < 0 || n < 0 || cRowOffset < 0 || cColOffset < 0) return OR_INVALID_PARAMETER;
  char *c0 = C ? (char *)C + elem_size(dtype) * ((size_t)cRowOffset + (size_t)cColOffset * ldc)
               : NULL;
  return oracle_gemm(dtype, opA, 0, m, n, kLocal, alpha, A, lda, B, ldb, beta, c0, ldc, NULL);
}

/*
 * Single-rank pgemm_sbs. gpu_order=0 follows the host entry
 * (src/pgemm_sbs/pgemm_sbs_host.cpp:175-183: no offset check on one rank),
 * gpu_order=1 the GPU entry (src/pgemm_sbs/pgemm_sbs_gpu.cpp:238-249).
 */
int oracle_pgemm_sbs(int dtype, int mLocal, int n, int k, const void *alpha, const void *A,
                     int lda, const void *B, int ldb, int bRowOffset, int bColOffset,
                     const void *beta, void *C, int ldc, int gpu_order) {
  if (k == 0 || n == 0) return OR_SUCCESS;
  if (gpu_order && (n < 0 || k < 0 || bRowOffset < 0 || bColOffset < 0))
    return OR_INVALID_PARAMETER;
  const char *b0 =
      B ? (const char *)B + elem_size(dtype) * ((size_t)bRowOffset + (size_t)bColOffset * ldb)
        : NULL;
  return oracle_gemm(dtype, 0, 0, mLocal, n, k, alpha, A, lda, b0, ldb, beta, C, ldc, NULL);
}

/* ---- block-cyclic index map (src/block_generation/block_cyclic_generator.cpp) ---- */

/* out[0..8] = globalRow, globalCol, globalSubRow, globalSubCol, localRow, localCol,
 * numRows, numCols, mpiRank for block `blockIdx` (column-major block order). */
void oracle_block_info(long rowsInBlock, long colsInBlock, long gridRows, long gridCols,
                       long globalNumRows, long globalNumCols, long rowOffset, long colOffset,
                       long blockIdx, long *out) {
  const long firstBlockRow = (rowOffset / rowsInBlock) * rowsInBlock;
  const long numBlockRows = (rowOffset - firstBlockRow + globalNumRows + rowsInBlock - 1) /
                            rowsInBlock;
  const long firstBlockCol = (colOffset / colsInBlock) * colsInBlock;
  const long bRow = blockIdx % numBlockRows;
  const long bCol = blockIdx / numBlockRows;
  const long gbRow = bRow + rowOffset / rowsInBlock;
  const long gbCol = bCol + colOffset / colsInBlock;
  long gRow = firstBlockRow + bRow * rowsInBlock;
  if (gRow < rowOffset) gRow = rowOffset;
  long gCol = firstBlockCol + bCol * colsInBlock;
  if (gCol < colOffset) gCol = colOffset;
  long endRow = (gbRow + 1) * rowsInBlock;
  if (endRow > rowOffset + globalNumRows) endRow = rowOffset + globalNumRows;
  long endCol = (gbCol + 1) * colsInBlock;
  if (endCol > colOffset + globalNumCols) endCol = colOffset + globalNumCols;
  out[0] = gRow;
  out[1] = gCol;
  out[2] = gRow - rowOffset;
  out[3] = gCol - colOffset;
  out[4] = (gbRow / gridRows) * rowsInBlock + gRow % rowsInBlock;
  out[5] = (gbCol / gridCols) * colsInBlock + gCol % colsInBlock;
  out[6] = endRow - gRow;
  out[7] = endCol - gCol;
  out[8] = (gbRow % gridRows) + (gbCol % gridCols) * gridRows;
}

long oracle_num_blocks(long rowsInBlock, long colsInBlock, long globalNumRows, long globalNumCols,
                       long rowOffset, long colOffset) {
  const long firstBlockRow = (rowOffset / rowsInBlock) * rowsInBlock;
  const long firstBlockCol = (colOffset / colsInBlock) * colsInBlock;
  const long nbr = (rowOffset - firstBlockRow + globalNumRows + rowsInBlock - 1) / rowsInBlock;
  const long nbc = (colOffset - firstBlockCol + globalNumCols + colsInBlock - 1) / colsInBlock;
  return nbr * nbc;
}

/* fill-mode predicate on a block (src/block_generation/block.hpp:58-66); mode 1 upper, 2 lower */
int oracle_block_is_active(long row, long col, long numRows, long numCols, long rowOffset,
                           long colOffset, int mode) {
  if (mode == 1) return col + numCols + colOffset > row + rowOffset;
  if (mode == 2) return row + numRows + rowOffset > col + colOffset;
  return 1;
}

/* rows/cols of a block-cyclic dimension held by process index procIdx
 * (src/block_generation/block_cyclic_generator.cpp:117-127) */
long oracle_local_size(long globalSize, long blockSize, long procIdx, long numProcs) {
  const long numBlocks = globalSize / blockSize;
  const long numOverhang = numBlocks % numProcs;
  long localSize = (numBlocks / numProcs) * blockSize;
  if (procIdx + 1 < numOverhang) localSize += blockSize;
  if (procIdx + 1 == numOverhang) localSize += globalSize % blockSize;
  return localSize;
}
