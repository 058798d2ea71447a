// The local GEMM engine: C <- alpha * op(A) * op(B) + beta * C on the
// context's GPU for any mix of host- and device-resident operands.
//
// Reference behaviour kept (src/gemm/gemm_gpu.cpp:59-174):
//   * the current device is the context's for the duration of the call;
//   * work already queued on the legacy default stream completes before the
//     operands are read (gemm_gpu.cpp:71-72);
//   * the call is synchronous: it returns when C is final;
//   * pointers are classified with cudaPointerGetAttributes; managed memory
//     counts as host memory (src/gpu_util/gpu_pointer_translation.hpp:39-81).
// Changed: there is no host-BLAS fallback for small problems (op_threshold_gpu
// is kept as a setting but every problem runs on the GPU), and host-resident
// A/B are streamed in k-chunks on a copy stream, double-buffered against the
// contraction on the compute stream, instead of being copied on the stream
// that consumes them (src/gpu_util/multiply_gpu.cpp:101-142).
#include <algorithm>
#include <cstring>

#include "../../../include/splab.h"
#include "internal.hpp"

namespace spla {

namespace {

template <typename T>
struct TypeCode;
template <>
struct TypeCode<float> {
  static constexpr int value = SPLAB_R32;
};
template <>
struct TypeCode<double> {
  static constexpr int value = SPLAB_R64;
};
template <>
struct TypeCode<std::complex<float>> {
  static constexpr int value = SPLAB_C32;
};
template <>
struct TypeCode<std::complex<double>> {
  static constexpr int value = SPLAB_C64;
};

bool is_device_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice;
}

struct DeviceGuard {
  int prev = 0;
  explicit DeviceGuard(int dev) {
    check_cuda(cudaGetDevice(&prev));
    if (prev != dev) check_cuda(cudaSetDevice(dev));
  }
  ~DeviceGuard() { cudaSetDevice(prev); }
};

int path_for(const ContextInternal& ctx, int) { return ctx.fp64_path(); }

// Copy the k-range [k0, k0 + kc) of an operand into a dense device buffer.
// `kmajor` operands have k as their contiguous (row) dimension: element
// (l, r) at X[l + r * ld] with r < rows; the others have element (r, l) at
// X[r + l * ld]. The dense copy keeps the same orientation with ld = kc
// (kmajor) or ld = rows (otherwise).
template <typename T>
void copy_k_chunk(T* dst, const T* src, int64_t ld, bool kmajor, int64_t rows, int64_t k0,
                  int64_t kc, cudaStream_t st) {
  const size_t es = sizeof(T);
  if (kmajor) {
    check_cuda(cudaMemcpy2DAsync(dst, kc * es, src + k0, ld * es, kc * es, rows,
                                 cudaMemcpyDefault, st));
  } else {
    check_cuda(cudaMemcpy2DAsync(dst, rows * es, src + k0 * ld, ld * es, rows * es, kc,
                                 cudaMemcpyDefault, st));
  }
}

}  // namespace

template <typename T>
void local_gemm(ContextInternal& ctx, SplaOperation opA, SplaOperation opB, int m, int n, int k,
                T alpha, const T* A, int lda, const T* B, int ldb, T beta, T* C, int ldc,
                SplaFillMode fill, int ro, int co) {
  if (m == 0 || n == 0) return;
  constexpr int dtype = TypeCode<T>::value;
  DeviceGuard guard(ctx.gpu_device_id());
  check_cuda(cudaStreamSynchronize(nullptr));  // API contract: default stream work is done

  if (lda < 1) lda = 1;
  if (ldb < 1) ldb = 1;
  if (ldc < m) throw InvalidParameterError();  // the reference hands this to BLAS unchecked
  const int path_pref = path_for(ctx, dtype);
  const int moduli = ctx.ozaki_moduli();
  cudaStream_t cs = ctx.compute_stream();

  const bool devA = k == 0 || is_device_pointer(A);
  const bool devB = k == 0 || is_device_pointer(B);
  const bool devC = is_device_pointer(C);

  // Device copy of C when C is host-resident (read only if beta != 0).
  T* dC = C;
  int64_t dldc = ldc;
  const bool beta_zero = beta == T(0);
  if (!devC) {
    dC = static_cast<T*>(ctx.device_pool().get(0, sizeof(T) * size_t(m) * n));
    dldc = m;
    if (!beta_zero)
      check_cuda(cudaMemcpy2DAsync(dC, size_t(m) * sizeof(T), C, size_t(ldc) * sizeof(T),
                                   size_t(m) * sizeof(T), n, cudaMemcpyDefault, cs));
  }

  if (devA && devB) {
    const int path = splab_gemm_path(dtype, path_pref, opA, opB, m, n, k);
    const size_t ws = splab_gemm_workspace_size(dtype, path, opA, opB, m, n, k, moduli);
    void* w = ws ? ctx.device_pool().get(1, ws) : nullptr;
    check_splab(splab_gemm(dtype, path, opA, opB, m, n, k, &alpha, A, lda, B, ldb, &beta, dC,
                           dldc, fill, ro, co, moduli, w, ws, cs));
    check_splab(splab_gemm_check(dtype, path, opA, opB, m, n, k, moduli, w, cs));
  } else {
    // Stream A and B in k-chunks: chunk c is copied on the copy stream into
    // buffer c % 2 while the compute stream contracts chunk c - 1; beta applies
    // to the first chunk only, later chunks accumulate (beta = 1).
    const bool akm = opA != SPLA_OP_NONE;  // A is k x m (k contiguous)
    const bool bkm = opB == SPLA_OP_NONE;  // B is k x n (k contiguous)
    const int64_t edge = std::max(64, ctx.tile_size_gpu());
    int64_t kc = std::max<int64_t>(256, (edge * edge * 4) / std::max(1, std::max(m, n)));
    kc = std::min<int64_t>(kc, k);
    kc = (kc + 63) / 64 * 64;
    if (kc > k) kc = k;
    const int64_t chunks = (k + kc - 1) / kc;
    const size_t abytes = sizeof(T) * size_t(kc) * m, bbytes = sizeof(T) * size_t(kc) * n;
    T* bufA[2] = {nullptr, nullptr};
    T* bufB[2] = {nullptr, nullptr};
    for (int b = 0; b < 2 && b < chunks; ++b) {
      if (!devA) bufA[b] = static_cast<T*>(ctx.device_pool().get(2 + b, abytes));
      if (!devB) bufB[b] = static_cast<T*>(ctx.device_pool().get(4 + b, bbytes));
    }
    const int64_t klast = k - (chunks - 1) * kc;
    const int path = splab_gemm_path(dtype, path_pref, opA, opB, m, n, kc);
    const size_t ws =
        std::max(splab_gemm_workspace_size(dtype, path, opA, opB, m, n, kc, moduli),
                 splab_gemm_workspace_size(dtype, path, opA, opB, m, n, klast, moduli));
    void* w = ws ? ctx.device_pool().get(1, ws) : nullptr;
    cudaStream_t xs = ctx.copy_stream();
    // C (if staged) must be in place before the first contraction
    check_cuda(cudaEventRecord(ctx.event(4), cs));
    check_cuda(cudaStreamWaitEvent(xs, ctx.event(4), 0));
    const T one = T(1);
    for (int64_t c = 0; c < chunks; ++c) {
      const int b = int(c % 2);
      const int64_t k0 = c * kc, kcur = std::min(kc, k - k0);
      if (c >= 2) check_cuda(cudaStreamWaitEvent(xs, ctx.event(2 + b), 0));  // buffer free
      const T* pa;
      int64_t la;
      if (devA) {
        pa = akm ? A + k0 : A + k0 * lda;
        la = lda;
      } else {
        copy_k_chunk(bufA[b], A, lda, akm, m, k0, kcur, xs);
        pa = bufA[b];
        la = akm ? kcur : m;
      }
      const T* pb;
      int64_t lb;
      if (devB) {
        pb = bkm ? B + k0 : B + k0 * ldb;
        lb = ldb;
      } else {
        copy_k_chunk(bufB[b], B, ldb, bkm, n, k0, kcur, xs);
        pb = bufB[b];
        lb = bkm ? kcur : n;
      }
      check_cuda(cudaEventRecord(ctx.event(b), xs));  // chunk ready
      check_cuda(cudaStreamWaitEvent(cs, ctx.event(b), 0));
      check_splab(splab_gemm(dtype, path, opA, opB, m, n, kcur, &alpha, pa, la, pb, lb,
                             c == 0 ? &beta : &one, dC, dldc, fill, ro, co, moduli, w, ws, cs));
      check_cuda(cudaEventRecord(ctx.event(2 + b), cs));  // buffer b consumed
    }
    check_splab(splab_gemm_check(dtype, path, opA, opB, m, n, klast, moduli, w, cs));
  }

  if (!devC)
    check_cuda(cudaMemcpy2DAsync(C, size_t(ldc) * sizeof(T), dC, size_t(m) * sizeof(T),
                                 size_t(m) * sizeof(T), n, cudaMemcpyDefault, cs));
  check_cuda(cudaStreamSynchronize(cs));
  check_cuda(cudaStreamSynchronize(ctx.copy_stream()));
}

template void local_gemm<float>(ContextInternal&, SplaOperation, SplaOperation, int, int, int,
                                float, const float*, int, const float*, int, float, float*, int,
                                SplaFillMode, int, int);
template void local_gemm<double>(ContextInternal&, SplaOperation, SplaOperation, int, int, int,
                                 double, const double*, int, const double*, int, double, double*,
                                 int, SplaFillMode, int, int);
template void local_gemm<std::complex<float>>(ContextInternal&, SplaOperation, SplaOperation, int,
                                              int, int, std::complex<float>,
                                              const std::complex<float>*, int,
                                              const std::complex<float>*, int,
                                              std::complex<float>, std::complex<float>*, int,
                                              SplaFillMode, int, int);
template void local_gemm<std::complex<double>>(ContextInternal&, SplaOperation, SplaOperation, int,
                                               int, int, std::complex<double>,
                                               const std::complex<double>*, int,
                                               const std::complex<double>*, int,
                                               std::complex<double>, std::complex<double>*, int,
                                               SplaFillMode, int, int);

}  // namespace spla
