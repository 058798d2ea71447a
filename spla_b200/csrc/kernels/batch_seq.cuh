// Batches on the tensor-core paths (Ozaki INT8, 3xTF32): the instances run one
// after another on one stream, sharing one workspace, and the whole sequence
// is replayed from a CUDA graph (batch_seq.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <vector>

#include "gemm_dmma.cuh"

namespace splab {

struct SeqBatch;
// path: SPLAB_PATH_OZAKI or SPLAB_PATH_TF32X3. Returns null when an instance
// is not supported by the path (dtype, op pair).
SeqBatch* seq_batch_create(int path, const std::vector<GemmProblem>& probs);
size_t seq_batch_workspace(const SeqBatch* b);
// First run executes the sequence directly; later runs capture it once (per
// workspace pointer) and replay the graph, ordered after `stream`.
cudaError_t seq_batch_run(SeqBatch* b, void* ws, cudaStream_t stream);
// Status of the last run (synchronises `stream`): 0 ok, 1 a bounded device
// wait gave up in one of the instances.
int seq_batch_status(SeqBatch* b, void* ws, cudaStream_t stream);
void seq_batch_destroy(SeqBatch* b);

}  // namespace splab
