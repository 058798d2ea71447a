// Shared device helpers for the sm_100a kernels of the SPLA local contraction.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace splab {

// Element type descriptors. Complex values are interleaved (re, im) pairs, the
// layout of std::complex / the reference's cuDoubleComplex reinterpretation
// (src/gpu_util/gpu_complex_type_conversion.hpp:40-84).
enum DType : int { kR32 = 0, kR64 = 1, kC32 = 2, kC64 = 3 };

__host__ __device__ constexpr bool dtype_is_complex(int d) { return d >= 2; }
__host__ __device__ constexpr bool dtype_is_double(int d) { return d == kR64 || d == kC64; }
__host__ __device__ constexpr int dtype_bytes(int d) {
  return d == kR32 ? 4 : (d == kC64 ? 16 : 8);
}

// 8- and 4-byte asynchronous global->shared copies with zero fill when
// `valid` is false (src-size 0 reads nothing).
__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem, bool valid) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_4(void* smem, const void* gmem, bool valid) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const int n = valid ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
// 16-byte asynchronous global->shared copy through L2 only (both addresses
// 16-byte aligned).
__device__ __forceinline__ void cp_async_16_cg(void* smem, const void* gmem) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Flip the sign bit of a double by mask (0 or 0x8000...): conjugation without
// spending FP64 pipe cycles.
__device__ __forceinline__ double xor_sign(double x, unsigned long long mask) {
  return __longlong_as_double(__double_as_longlong(x) ^ mask);
}

// Fill-mode activity of a tile of C, the predicate of the reference's
// block_is_active (src/block_generation/block.hpp:58-66) applied to the tile
// at local (row, col) of size rows x cols with the C offsets (ro, co).
// mode: 0 full, 1 upper, 2 lower.
__host__ __device__ __forceinline__ bool tile_is_active(int mode, int64_t row, int64_t col,
                                                        int64_t rows, int64_t cols, int64_t ro,
                                                        int64_t co) {
  if (mode == 1) return col + cols + co > row + ro;
  if (mode == 2) return row + rows + ro > col + co;
  return true;
}

// Phase events set by splab_set_phase_events (per host thread).
struct PhaseEvents {
  cudaEvent_t* ev = nullptr;
  int count = 0;
};
PhaseEvents& phase_events();

// cudaFuncAttributeMaxDynamicSharedMemorySize of `func` on the current device,
// set once per device (thread-safe); returns the CUDA status of that call.
cudaError_t set_dynamic_smem(const void* func, int bytes);
inline void phase_mark(int phase, bool end, cudaStream_t st) {
  PhaseEvents& pe = phase_events();
  if (pe.ev && phase < pe.count &&
      cudaEventRecord(pe.ev[2 * phase + (end ? 1 : 0)], st) != cudaSuccess)
    cudaGetLastError();  // a bad timing event must not fail the computation
}

}  // namespace splab
