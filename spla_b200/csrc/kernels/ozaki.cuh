// Host-side interface of the Ozaki scheme II contraction (ozaki.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "gemm_dmma.cuh"

namespace splab {

// Device scratch needed by ozaki_gemm for this problem with `moduli` CRT
// moduli (0 = default).
size_t ozaki_workspace_bytes(const GemmProblem& prob, int moduli);

// C <- alpha * op(A) * op(B) + beta * C for double / complex double through
// INT8 residue GEMMs on tcgen05 and Chinese-remainder reconstruction.
cudaError_t ozaki_gemm(const GemmProblem& prob, int moduli, void* workspace, size_t ws_bytes,
                       cudaStream_t stream);

}  // namespace splab
