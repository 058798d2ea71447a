// Host-side interface of the 3xTF32 contraction for float / complex float
// (tf32x3.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "gemm_dmma.cuh"

namespace splab {

// True when the 3xTF32 path handles this problem: float or complex float,
// op(A) in {T, C}, op(B) = N.
bool tf32x3_supported(const GemmProblem& prob);

// Device scratch needed by tf32x3_gemm (hi/lo operand planes, FP64 partials).
size_t tf32x3_workspace_bytes(const GemmProblem& prob);

// C <- alpha * op(A) * B + beta * C with each float split into two TF32
// parts and three TF32 tensor-core products per pair of elements.
cudaError_t tf32x3_gemm(const GemmProblem& prob, void* workspace, size_t ws_bytes,
                        cudaStream_t stream);

// Status word of the last tf32x3_gemm on this workspace (synchronises
// `stream`): 0 = ok, 1 = a bounded device wait gave up.
int tf32x3_status(const GemmProblem& prob, void* workspace, cudaStream_t stream);

// Device address of the status word inside the workspace.
int* tf32x3_status_ptr(const GemmProblem& prob, void* workspace);

}  // namespace splab
