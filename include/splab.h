/*
 * splab: the kernel-level C ABI of the B200 implementation of SPLA's local
 * contraction. Plain pointers, 64-bit sizes and a CUDA stream (passed as
 * void*); no allocation inside except where stated; never throws. The SPLA
 * host layer (spla_* in include/spla/) validates arguments, manages memory
 * and calls these. Each entry point names the reference interface whose
 * work it performs.
 *
 * Conventions
 *   dtype : SPLAB_R32, SPLAB_R64, SPLAB_C32, SPLAB_C64 (complex interleaved re,im)
 *   op    : 0 = none, 1 = transpose, 2 = conjugate transpose (SplaOperation)
 *   alpha, beta : HOST pointers to one scalar of the dtype (complex: 2 values)
 *   A, B, C     : DEVICE pointers, column-major with leading dimensions lda/ldb/ldc
 *   fill        : 0 full, 1 upper, 2 lower; tiles of C that do not intersect
 *                 the triangle (with C's offsets ro/co in the distributed
 *                 matrix) are skipped and left unchanged
 *   workspace   : DEVICE scratch of at least splab_gemm_workspace_size() bytes
 *   Return value: SPLAB_OK or an SPLAB_ERR_* code (splab_status_string()).
 */
#ifndef SPLAB_H
#define SPLAB_H
#include <stddef.h>
#include <stdint.h>

#ifndef SPLAB_API
#define SPLAB_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SPLAB_R32 0
#define SPLAB_R64 1
#define SPLAB_C32 2
#define SPLAB_C64 3

/* Compute paths for the contraction. */
#define SPLAB_PATH_AUTO 0  /* the supported path with the least modelled time */
#define SPLAB_PATH_DMMA 1  /* FP64 tensor cores (mma.sync f64); float inputs accumulate in FP64 */
#define SPLAB_PATH_OZAKI 2 /* Ozaki scheme II on INT8 tcgen05 (all four dtypes), any
                              op pair: op(A) = N and op(B) in {T, C} are read in place
                              (conjugated on load for C) */
#define SPLAB_PATH_TF32X3 3 /* float / complex float: each input split into two TF32
                               parts, three TF32 tcgen05 products, FP32 accumulation
                               in 64-real windows folded into double-float sums; any
                               op pair: op(A) = N and op(B) in {T, C} are first copied
                               k-major into the workspace (conjugated for C); double
                               dtypes use DMMA */

#define SPLAB_OK 0
#define SPLAB_ERR_INVALID 1     /* bad argument (sizes, leading dimensions, dtype, path) */
#define SPLAB_ERR_WORKSPACE 2   /* workspace missing or too small */
#define SPLAB_ERR_LAUNCH 3      /* a CUDA launch or runtime call failed */
#define SPLAB_ERR_UNSUPPORTED 4 /* path not available for this dtype / device */
#define SPLAB_ERR_TIMEOUT 5     /* a bounded device-side wait gave up */

SPLAB_API const char *splab_status_string(int status);

/* The concrete path (SPLAB_PATH_DMMA, SPLAB_PATH_OZAKI or SPLAB_PATH_TF32X3)
 * `path` resolves to for this problem. An explicit path resolves to itself when
 * it supports the problem, else to DMMA. SPLAB_PATH_AUTO picks, among the
 * supported paths whose workspace fits in a quarter of the device memory, the
 * one with the least modelled time (a model of each path measured on B200;
 * a tensor-core path must beat DMMA by 10 %). The result depends only on the
 * problem and the device. */
SPLAB_API int splab_gemm_path(int dtype, int path, int opA, int opB, int64_t m, int64_t n,
                              int64_t k);

/* Bytes of device scratch splab_gemm needs for this problem (0 if none);
 * ozakiModuli as for splab_gemm. */
SPLAB_API size_t splab_gemm_workspace_size(int dtype, int path, int opA, int opB, int64_t m,
                                           int64_t n, int64_t k, int ozakiModuli);

/*
 * C <- alpha * op(A) * op(B) + beta * C on the device, asynchronous on `stream`.
 * Performs the local work of spla_?gemm (reference src/gemm/gemm_gpu.cpp:59-174
 * and src/gpu_util/multiply_gpu.cpp:78-143), which the single-rank pgemm_ssb
 * (src/pgemm_ssb/pgemm_ssb_gpu.cpp:259-262, opA in {T,C}, opB = N) and
 * pgemm_sbs (src/pgemm_sbs/pgemm_sbs_gpu.cpp:246-249, N,N) reduce to, plus the
 * fill-mode tile skipping of pgemm_ssbtr (src/block_generation/block.hpp:58-66).
 * ozakiModuli: number of CRT moduli for SPLAB_PATH_OZAKI (0 = default: 15 for
 * double, <= 1e-14 relative error; 9 for float, ~1e-8; range 8..16); ignored
 * otherwise. A bounded device wait
 * that gives up makes the next splab_gemm_check() return SPLAB_ERR_TIMEOUT.
 */
SPLAB_API int splab_gemm(int dtype, int path, int opA, int opB, int64_t m, int64_t n, int64_t k,
               const void *alpha, const void *A, int64_t lda, const void *B, int64_t ldb,
               const void *beta, void *C, int64_t ldc, int fill, int64_t ro, int64_t co,
               int ozakiModuli, void *workspace, size_t workspaceBytes, void *stream);

/*
 * Synchronise `stream` and report a device-side failure of the last
 * splab_gemm that used `workspace` (SPLAB_OK or SPLAB_ERR_TIMEOUT).
 */
SPLAB_API int splab_gemm_check(int dtype, int path, int opA, int opB, int64_t m, int64_t n,
                               int64_t k, int ozakiModuli, void *workspace, void *stream);

/*
 * Allocation-free FP64 contraction (no counterpart in the reference library).
 *
 * Same operation and arguments as splab_gemm on the DMMA path (FP64 tensor
 * cores), minus the workspace: for callers that cannot allocate device
 * memory - applications whose device memory belongs to a framework allocator
 * that must account for every byte, processes under a hard device-memory
 * cap, and latency-critical loops that cannot take the device synchronisation
 * of cudaMalloc / cudaFree. It allocates nothing: the split-K partials live
 * in one static device array of SPLAB_NOALLOC_SCRATCH_BYTES (64 MiB) that
 * every GPU loading the library holds until exit. A problem that splab_gemm
 * would run with one k-split (small k, or k = 0) needs no partials and runs at
 * any size. One that splab_gemm splits along k needs one FP64 partial of C
 * per split, m * n * e bytes (e = 16 for complex, 8 for real dtypes): it runs
 * with as many splits as fit in the array (fewer than splab_gemm when needed)
 * and is rejected with SPLAB_ERR_WORKSPACE when not even two fit
 * (m * n * e > 32 MiB). The first call on a device, and the first after a
 * device reset, looks up the array's device address (with that device
 * current); make that first call before any stream capture. All calls share
 * the array: calls that overlap on the GPU race and must be serialised by the
 * caller. Inputs and outputs are passed by the caller as for splab_gemm;
 * alpha/beta are host pointers.
 */
#define SPLAB_NOALLOC_SCRATCH_BYTES (64u << 20)
SPLAB_API int splab_gemm_dmma_noalloc(int dtype, int opA, int opB, int64_t m, int64_t n, int64_t k,
                                      const void *alpha, const void *A, int64_t lda,
                                      const void *B, int64_t ldb, const void *beta, void *C,
                                      int64_t ldc, int fill, int64_t ro, int64_t co,
                                      void *stream);

/*
 * Batched grouped contraction (the many-instance form of splab_gemm): all
 * problems share dtype and op(A)/op(B); each has its own sizes, pointers,
 * alpha and beta (as (re, im) doubles; im ignored for real dtypes). One
 * persistent launch walks every (problem, tile, k-chunk) work item, one
 * grouped launch reduces the split-K partials; the pair is captured in a CUDA
 * graph on the first run and replayed afterwards. The CTA tile and the
 * k-chunk size are chosen by measuring every candidate pair on the first run
 * (autotune != 0; C is not written while measuring) or by a model otherwise. FP64 tensor-core path
 * (float inputs accumulate in FP64). No counterpart in the reference library
 * (a batch there is a loop of pgemm_ssb calls).
 */
typedef struct splab_problem {
  int opA, opB;
  int64_t m, n, k;
  const void *A;
  int64_t lda;
  const void *B;
  int64_t ldb;
  void *C;
  int64_t ldc;
  double alpha[2], beta[2];
} splab_problem;

SPLAB_API int splab_batch_create(int dtype, int count, const splab_problem *problems,
                                 void **plan, size_t *workspaceBytes);
/* The same batch on a chosen path: SPLAB_PATH_DMMA or SPLAB_PATH_AUTO give the
 * grouped FP64 launch above; SPLAB_PATH_OZAKI (any dtype) and
 * SPLAB_PATH_TF32X3 (float dtypes) run the instances one after another on one
 * stream with one shared workspace (the largest instance's), the sequence
 * captured in a CUDA graph on the second run and replayed afterwards.
 * SPLAB_ERR_UNSUPPORTED when an instance's dtype or op pair is not handled by
 * the path (Ozaki: every op pair; 3x TF32 batches: op(A) in {T, C}, op(B) = N,
 * the k-major copies of splab_gemm being made per call). */
SPLAB_API int splab_batch_create_path(int dtype, int path, int count,
                                      const splab_problem *problems, void **plan,
                                      size_t *workspaceBytes);
/* Run (and on the first call tune + capture) the batch on `stream`; workspace
 * must hold workspaceBytes of device memory and stay the same between runs
 * (a different pointer triggers a new capture). */
SPLAB_API int splab_batch_run(void *plan, void *workspace, size_t workspaceBytes, int autotune,
                              void *stream);
/* Chosen k-chunk; the k-chunk and measured time (ms) of each tuning entry
 * (one per tile configuration and k-chunk) when tuned, else the candidate
 * k-chunks with time -1; arrays of at least 32 entries. */
SPLAB_API int splab_batch_info(void *plan, int64_t *kChunk, int *nCandidates, int64_t *candidates,
                               double *tuningMs);
/* CTA tile chosen for the grouped FP64 launch, and per tuning entry (the
 * entries of splab_batch_info, arrays of at least 32) the tile it measured;
 * the autotuner tries each k-chunk with the default tile (complex 64x64,
 * real 128x64) and a larger one (complex 128x64, real 128x128). Zero for the
 * tensor-core paths. */
SPLAB_API int splab_batch_tiles(void *plan, int *tileM, int *tileN, int *nEntries,
                                int *entryTileM, int *entryTileN);
/* Synchronise `stream` and report SPLAB_ERR_TIMEOUT when a bounded device wait
 * gave up in the last run of a tensor-core batch (SPLAB_OK otherwise). */
SPLAB_API int splab_batch_check(void *plan, void *workspace, void *stream);
SPLAB_API int splab_batch_destroy(void *plan);

/*
 * Block-cyclic index map on the device: for each of `count` block indices in
 * blockIdx (device, column-major block order) write 9 int64 values to out
 * (device): global row, global col, global sub-row, global sub-col, local row,
 * local col, rows, cols, owning rank. Same mapping as the reference's
 * BlockCyclicGenerator::get_block_info
 * (src/block_generation/block_cyclic_generator.cpp:59-100).
 */
SPLAB_API int splab_block_cyclic_info(int64_t rowsInBlock, int64_t colsInBlock, int64_t gridRows,
                            int64_t gridCols, int64_t globalRows, int64_t globalCols,
                            int64_t rowOffset, int64_t colOffset, const int64_t *blockIdx,
                            int64_t count, int64_t *out, void *stream);

/*
 * Multi-rank exchange support (pgemm_ssb / pgemm_sbs over several ranks).
 *
 * splab_block_cyclic_blocks: HOST. The block-cyclic map of the
 * globalRows x globalCols submatrix at (rowOffset, colOffset) of a matrix in
 * rowsInBlock x colsInBlock blocks on a gridRows x gridCols process grid, as
 * BlockCyclicGenerator::get_block_info does it
 * (src/block_generation/block_cyclic_generator.cpp:59-100): returns the
 * number of blocks (-1 on bad arguments) and, when out is non-null, writes 9
 * values per block (global row, global col, sub-row, sub-col, local row,
 * local col, rows, cols, grid index of the owner) in column-major block
 * order. The exchange plans of the distributed layer are built from it.
 *
 * splab_copy_blocks: DEVICE, asynchronous on `stream`. For each of `count`
 * block descriptors (6 int64 in device memory: srcOff, srcLd, dstOff, dstLd,
 * rows, cols, in elements) dst[dstOff + i + j*dstLd] =
 * alpha * src[srcOff + i + j*srcLd] + beta * dst[...] (dst not read when beta
 * is 0); maxBlockElems bounds rows*cols. src, dst and desc must be memory the
 * device can reach (SPLAB_ERR_INVALID otherwise); the descriptors must stay
 * inside the buffers. alpha/beta are host scalars of the
 * dtype. It performs the block moves of the reference's ring engines: sending
 * each finished block of C to its owner and adding it there
 * (src/pgemm_ssb/ring_ssb_gpu.cpp:413-500, src/pgemm_ssb/add_kernel.cpp:40-62)
 * and redistributing the blocks of B (src/pgemm_sbs/ring_sbs_gpu.cpp:114-351).
 */
SPLAB_API int64_t splab_block_cyclic_blocks(int64_t rowsInBlock, int64_t colsInBlock,
                                            int64_t gridRows, int64_t gridCols,
                                            int64_t globalRows, int64_t globalCols,
                                            int64_t rowOffset, int64_t colOffset, int64_t *out);
SPLAB_API int splab_copy_blocks(int dtype, const void *src, void *dst, const int64_t *desc,
                                int64_t count, int64_t maxBlockElems, const void *alpha,
                                const void *beta, void *stream);

/*
 * Double-double reference product for verification (no reference counterpart;
 * it is the device form of the compensated CPU oracle and sits on no
 * contraction path): R = op(A) * op(B) with every product split exactly
 * (TwoProduct) and summed with TwoSum (Ogita-Rump-Oishi Dot2), as accurate as
 * a dot product in twice the working precision. A and B of any dtype (read
 * as double); Rhi and, when non-null, Rlo are DEVICE double buffers (complex:
 * interleaved re, im) with leading dimension ldr in elements. Asynchronous
 * on `stream`. Lets results be checked on the whole C at full problem sizes.
 */
SPLAB_API int splab_gemm_dd(int dtype, int opA, int opB, int64_t m, int64_t n, int64_t k,
                            const void *A, int64_t lda, const void *B, int64_t ldb, double *Rhi,
                            double *Rlo, int64_t ldr, void *stream);

/*
 * Phase timing for measurement harnesses (no reference counterpart). When
 * `events` is non-null, every following splab_gemm on the calling host thread
 * records events[2p] / events[2p+1] (cudaEvent_t handles created by the
 * caller) on its stream around phase p, for p < count:
 *   DMMA path : 0 = contraction kernel, 1 = split-K reduction
 *   Ozaki path: 0 = slicing, 1 = INT8 residue GEMMs, 2 = reconstruction,
 *               3 + g = GEMM launch of modulus group g; inside phase 0:
 *               15 = k-major copy of A (op(A) = N with k too long to be read in
 *               place), 16 = row norms (of A, and
 *               of B unless they run on a side stream), 17 = residues of A,
 *               18 = residues of B (one modulus group)
 * Pass events = NULL to stop. Returns SPLAB_OK.
 */
SPLAB_API int splab_set_phase_events(void **events, int count);

#ifdef __cplusplus
}
#endif
#endif
