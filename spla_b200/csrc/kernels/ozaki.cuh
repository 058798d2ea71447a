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

// C <- alpha * op(A) * op(B) + beta * C for the four dtypes through INT8
// residue GEMMs on tcgen05 and Chinese-remainder reconstruction.
// True when the Ozaki path handles this problem: any op(A); op(B) = N, or
// op(B) in {T, C} read in place (k within the transposing slicer's grid);
// m <= 2^24, n <= 2^23.
bool ozaki_supported(const GemmProblem& prob);

// True when op(A) = N is too long along k to be read in place, so that A is
// first copied k-major into the workspace.
bool ozaki_copies_a(const GemmProblem& prob);

// Status word of the last ozaki_gemm on this workspace (synchronises
// `stream`): 0 = ok, 1 = a bounded device wait gave up.
int ozaki_status(const GemmProblem& prob, int moduli, void* workspace, cudaStream_t stream);

cudaError_t ozaki_gemm(const GemmProblem& prob, int moduli, void* workspace, size_t ws_bytes,
                       cudaStream_t stream);

// Device address of the status word inside the workspace.
int* ozaki_status_ptr(const GemmProblem& prob, int moduli, void* workspace);

// Whether ozaki_gemm may use its side streams on this host thread (default
// yes); a batch turns them off while it captures a CUDA graph on one stream.
void ozaki_allow_side_streams(bool allow);

}  // namespace splab
