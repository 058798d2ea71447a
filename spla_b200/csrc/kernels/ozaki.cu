// Ozaki scheme II contraction (placeholder until the tcgen05 kernels land).
#include "ozaki.cuh"

namespace splab {
size_t ozaki_workspace_bytes(const GemmProblem&, int) { return 0; }
cudaError_t ozaki_gemm(const GemmProblem&, int, void*, size_t, cudaStream_t) {
  return cudaErrorNotSupported;
}
}  // namespace splab
