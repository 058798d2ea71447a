// Host-side interface of the FP64 tensor-core contraction (gemm_dmma.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace splab {

// One local GEMM  C <- alpha * op(A) * op(B) + beta * C  (column-major).
struct GemmProblem {
  int dtype;     // DType
  int opA, opB;  // 0 = N, 1 = T, 2 = C (SplaOperation values)
  int64_t m, n, k;
  const void* A;
  int64_t lda;
  const void* B;
  int64_t ldb;
  void* C;
  int64_t ldc;
  double alpha[2], beta[2];  // (re, im); im = 0 for real dtypes
  int fill_mode;             // 0 full, 1 upper, 2 lower (tiles outside are skipped)
  int64_t fill_ro, fill_co;  // offsets of C inside the distributed matrix
};

struct DmmaParams {
  const void* A;
  const void* B;
  void* C;
  void* P;  // split-K partials, [split][n][m], FP64 (complex: double2)
  int64_t lda, ldb, ldc, m, n, k, k_per_split;
  double alpha_r, alpha_i, beta_r, beta_i;
  int conj_a, conj_b, partial, fill_mode;
  int64_t fill_ro, fill_co;
};

// Launch plan chosen for a problem: tile sizes, split count, workspace.
struct DmmaPlan {
  int bm, bn, splits;
  int64_t k_per_split;
  size_t workspace_bytes;
};

DmmaPlan dmma_plan(const GemmProblem& prob, int num_sms, int force_splits = 0);
cudaError_t dmma_gemm(const GemmProblem& prob, const DmmaPlan& plan, void* workspace,
                      cudaStream_t stream);

// The DMMA contraction with its split-K partials in a static device array
// (no allocation). Returns 0, 2 when the problem needs more scratch than the
// array holds, 3 on a CUDA error.
int dmma_gemm_noalloc(const GemmProblem& prob, int num_sms, cudaStream_t stream);

// Batched grouped FP64 contraction (one dtype and operand layout per batch).
struct BatchPlanImpl;
BatchPlanImpl* batch_create(int dtype, const std::vector<GemmProblem>& probs);
size_t batch_workspace(const BatchPlanImpl* plan);
// First run measures every (CTA tile configuration, k-chunk) pair (autotune)
// or takes the model choice, then captures the grouped launch in a CUDA graph;
// later runs replay.
cudaError_t batch_run(BatchPlanImpl* plan, void* workspace, cudaStream_t stream, bool autotune);
void batch_destroy(BatchPlanImpl* plan);
int64_t batch_kc(const BatchPlanImpl* plan);
const std::vector<double>& batch_tuning(const BatchPlanImpl* plan);
// The k-chunk of each tuning entry after an autotuned first run (the
// candidate k-chunks before it).
const std::vector<int64_t>& batch_candidates(const BatchPlanImpl* plan);
// Chosen CTA tile and the tile of each tuning entry.
void batch_tiles(const BatchPlanImpl* plan, int* bm, int* bn, std::vector<int>* entry_bm,
                 std::vector<int>* entry_bn);

// Sum `splits` FP64 partial tiles in order and apply alpha/beta into C.
cudaError_t reduce_partials(const GemmProblem& prob, const void* partials, int splits, int tile_m,
                            int tile_n, cudaStream_t stream);

}  // namespace splab
