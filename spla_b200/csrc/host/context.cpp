// spla::Context and the spla_ctx_* C ABI (reference include/spla/context.h,
// src/spla/context.cpp, src/spla/context_internal.hpp). Defaults and setter
// validation equal the reference's (context_internal.hpp:58-64, :122-140).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../../include/splab.h"
#include "internal.hpp"
#include "spla/context.h"

namespace spla {

void check_cuda(cudaError_t err) {
  if (err == cudaSuccess) return;
  if (std::getenv("SPLA_B200_DEBUG"))
    std::fprintf(stderr, "spla_b200: CUDA error %s (%s)\n", cudaGetErrorName(err),
                 cudaGetErrorString(err));
  cudaGetLastError();  // clear a sticky-free error so the context stays usable
  switch (err) {
    case cudaErrorMemoryAllocation: throw GPUAllocationError();
    case cudaErrorLaunchFailure:
    case cudaErrorLaunchOutOfResources:
    case cudaErrorLaunchTimeout:
    case cudaErrorInvalidConfiguration: throw GPULaunchError();
    case cudaErrorNoDevice: throw GPUNoDeviceError();
    case cudaErrorInvalidValue: throw GPUInvalidValueError();
    case cudaErrorInvalidDevicePointer: throw GPUInvalidDevicePointerError();
    default: throw GPUError();
  }
}

void check_splab(int status) {
  if (status != SPLAB_OK && std::getenv("SPLA_B200_DEBUG"))
    std::fprintf(stderr, "spla_b200: splab status %d (%s), last CUDA error %s\n", status,
                 splab_status_string(status), cudaGetErrorName(cudaPeekAtLastError()));
  switch (status) {
    case SPLAB_OK: return;
    case SPLAB_ERR_INVALID: throw InvalidParameterError();
    case SPLAB_ERR_WORKSPACE: throw InternalError();
    case SPLAB_ERR_LAUNCH: throw GPULaunchError();
    case SPLAB_ERR_UNSUPPORTED: throw GPUSupportError();
    case SPLAB_ERR_TIMEOUT: throw GPULaunchError();
    default: throw GenericError();
  }
}

void* ScratchPool::get(int slot, std::size_t bytes) {
  if (slot < 0 || slot >= kSlots) throw InternalError();
  if (bytes == 0) bytes = 256;
  if (size_[slot] >= bytes) return ptr_[slot];
  if (ptr_[slot]) {
    if (kind_ != kHost) cudaDeviceSynchronize();  // the old buffer may still be in use
    free_(ptr_[slot]);
    held_ -= size_[slot];
    ptr_[slot] = nullptr;
    size_[slot] = 0;
  }
  // grow with headroom so that slightly larger calls do not reallocate
  const std::size_t want = bytes + bytes / 8;
  void* p = alloc_(want);
  if (!p) {
    if (kind_ == kDevice) throw GPUAllocationError();
    if (kind_ == kPinned) throw GPUAllocationError();
    throw MPIAllocError();
  }
  ptr_[slot] = p;
  size_[slot] = want;
  held_ += want;
  return p;
}

void ScratchPool::release() {
  for (int i = 0; i < kSlots; ++i) {
    if (ptr_[i]) {
      if (kind_ != kHost) cudaDeviceSynchronize();
      free_(ptr_[i]);
    }
    ptr_[i] = nullptr;
    size_[i] = 0;
  }
  held_ = 0;
}

namespace {
int path_from_env() {
  const char* v = std::getenv("SPLA_B200_PATH");
  if (!v) return SPLAB_PATH_AUTO;
  if (!std::strcmp(v, "dmma")) return SPLAB_PATH_DMMA;
  if (!std::strcmp(v, "ozaki")) return SPLAB_PATH_OZAKI;
  if (!std::strcmp(v, "tf32x3")) return SPLAB_PATH_TF32X3;
  return SPLAB_PATH_AUTO;
}
}  // namespace

ContextInternal::ContextInternal(SplaProcessingUnit pu)
    : pu_(pu), tileSizeHost_(pu == SPLA_PU_HOST ? 500 : 1500) {
  if (pu != SPLA_PU_HOST && pu != SPLA_PU_GPU) throw InvalidParameterError();
  int count = 0;
  const cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count < 1) {
    cudaGetLastError();
    // A host context is created without touching a device, as the
    // reference's (context_internal.hpp:58-73: device id 0); its
    // contractions, which run on the GPU here, report the missing device.
    if (pu != SPLA_PU_HOST) throw GPUNoDeviceError();
  } else {
    check_cuda(cudaGetDevice(&deviceId_));
    hasDevice_ = true;
  }
  fp64Path_ = path_from_env();
  if (const char* v = std::getenv("SPLA_B200_OZAKI_MODULI")) {
    const int m = std::atoi(v);  // valid: 8 .. 16; anything else keeps the default
    if (m >= 8 && m <= 16) ozakiModuli_ = m;
  }
  host_.reset(new ScratchPool(ScratchPool::kHost, std::malloc, std::free));
  pinned_.reset(new ScratchPool(
      ScratchPool::kPinned,
      [](std::size_t s) -> void* {
        void* p = nullptr;
        return cudaMallocHost(&p, s) == cudaSuccess ? p : nullptr;
      },
      [](void* p) { cudaFreeHost(p); }));
  device_.reset(new ScratchPool(
      ScratchPool::kDevice,
      [](std::size_t s) -> void* {
        void* p = nullptr;
        return cudaMalloc(&p, s) == cudaSuccess ? p : nullptr;
      },
      [](void* p) { cudaFree(p); }));
}

ContextInternal::~ContextInternal() {
  if (!hasDevice_) return;  // nothing was allocated or created on a device
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(deviceId_);
  if (compute_) cudaStreamSynchronize(compute_);
  if (copy_) cudaStreamSynchronize(copy_);
  device_.reset();
  pinned_.reset();
  host_.reset();
  for (auto& ev : events_)
    if (ev) cudaEventDestroy(ev);
  if (compute_) cudaStreamDestroy(compute_);
  if (copy_) cudaStreamDestroy(copy_);
  cudaSetDevice(prev);
}

cudaStream_t ContextInternal::compute_stream() {
  if (!compute_) check_cuda(cudaStreamCreateWithFlags(&compute_, cudaStreamNonBlocking));
  return compute_;
}

cudaStream_t ContextInternal::copy_stream() {
  if (!copy_) check_cuda(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
  return copy_;
}

cudaEvent_t ContextInternal::event(int i) {
  if (i < 0 || i >= 8) throw InternalError();
  if (!events_[i]) check_cuda(cudaEventCreateWithFlags(&events_[i], cudaEventDisableTiming));
  return events_[i];
}

// ---------------------------------------------------------------------------
// spla::Context

Context::Context(SplaProcessingUnit pu) : ctxInternal_(new ContextInternal(pu)) {}
SplaProcessingUnit Context::processing_unit() const { return ctxInternal_->processing_unit(); }
int Context::num_tiles() const { return ctxInternal_->num_tiles(); }
int Context::tile_size_host() const { return ctxInternal_->tile_size_host(); }
int Context::tile_size_gpu() const { return ctxInternal_->tile_size_gpu(); }
int Context::op_threshold_gpu() const { return ctxInternal_->op_threshold_gpu(); }
int Context::gpu_device_id() const { return ctxInternal_->gpu_device_id(); }
std::uint_least64_t Context::allocated_memory_host() const {
  return ctxInternal_->host_pool().bytes_held();
}
std::uint_least64_t Context::allocated_memory_pinned() const {
  return ctxInternal_->pinned_pool().bytes_held();
}
std::uint_least64_t Context::allocated_memory_gpu() const {
  return ctxInternal_->device_pool().bytes_held();
}
void Context::set_num_tiles(int v) { ctxInternal_->set_num_tiles(v); }
void Context::set_tile_size_host(int v) { ctxInternal_->set_tile_size_host(v); }
void Context::set_op_threshold_gpu(int v) { ctxInternal_->set_op_threshold_gpu(v); }
void Context::set_tile_size_gpu(int v) { ctxInternal_->set_tile_size_gpu(v); }
void Context::set_alloc_host(std::function<void*(std::size_t)> a, std::function<void(void*)> f) {
  if (!a || !f) throw InvalidAllocatorFunctionError();
  ctxInternal_->host_pool().set_functions(std::move(a), std::move(f));
}
void Context::set_alloc_pinned(std::function<void*(std::size_t)> a, std::function<void(void*)> f) {
  if (!a || !f) throw InvalidAllocatorFunctionError();
  ctxInternal_->pinned_pool().set_functions(std::move(a), std::move(f));
}
void Context::set_alloc_gpu(std::function<void*(std::size_t)> a, std::function<void(void*)> f) {
  if (!a || !f) throw InvalidAllocatorFunctionError();
  ctxInternal_->device_pool().set_functions(std::move(a), std::move(f));
}

}  // namespace spla

// ---------------------------------------------------------------------------
// C ABI (reference src/spla/context.cpp:120-366). Null handles return
// SPLA_INVALID_HANDLE_ERROR.

namespace {
template <typename F>
SplaError guarded(F&& f) {
  try {
    f();
  } catch (const spla::GenericError& e) {
    return e.error_code();
  } catch (...) {
    return SPLA_UNKNOWN_ERROR;
  }
  return SPLA_SUCCESS;
}
spla::Context& as_ctx(SplaContext c) { return *static_cast<spla::Context*>(c); }
}  // namespace

extern "C" {

SplaError spla_ctx_create(SplaContext* ctx, SplaProcessingUnit pu) {
  if (!ctx) return SPLA_INVALID_POINTER_ERROR;
  return guarded([&] { *ctx = new spla::Context(pu); });
}

SplaError spla_ctx_destroy(SplaContext* ctx) {
  if (!ctx || !*ctx) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] {
    delete static_cast<spla::Context*>(*ctx);
    *ctx = nullptr;
  });
}

#define SPLA_B200_CTX_GETTER(NAME, TYPE, EXPR)                 \
  SplaError NAME(SplaContext ctx, TYPE* out) {                 \
    if (!ctx) return SPLA_INVALID_HANDLE_ERROR;                \
    return guarded([&] { *out = as_ctx(ctx).EXPR(); });        \
  }

SPLA_B200_CTX_GETTER(spla_ctx_processing_unit, SplaProcessingUnit, processing_unit)
SPLA_B200_CTX_GETTER(spla_ctx_num_tiles, int, num_tiles)
SPLA_B200_CTX_GETTER(spla_ctx_tile_size_host, int, tile_size_host)
SPLA_B200_CTX_GETTER(spla_ctx_tile_size_gpu, int, tile_size_gpu)
SPLA_B200_CTX_GETTER(spla_ctx_op_threshold_gpu, int, op_threshold_gpu)
SPLA_B200_CTX_GETTER(spla_ctx_gpu_device_id, int, gpu_device_id)
SPLA_B200_CTX_GETTER(spla_ctx_allocated_memory_host, uint_least64_t, allocated_memory_host)
SPLA_B200_CTX_GETTER(spla_ctx_allocated_memory_pinned, uint_least64_t, allocated_memory_pinned)
SPLA_B200_CTX_GETTER(spla_ctx_allocated_memory_gpu, uint_least64_t, allocated_memory_gpu)
#undef SPLA_B200_CTX_GETTER

#define SPLA_B200_CTX_SETTER(NAME, EXPR)                       \
  SplaError NAME(SplaContext ctx, int v) {                     \
    if (!ctx) return SPLA_INVALID_HANDLE_ERROR;                \
    return guarded([&] { as_ctx(ctx).EXPR(v); });              \
  }

SPLA_B200_CTX_SETTER(spla_ctx_set_num_tiles, set_num_tiles)
SPLA_B200_CTX_SETTER(spla_ctx_set_tile_size_host, set_tile_size_host)
SPLA_B200_CTX_SETTER(spla_ctx_set_op_threshold_gpu, set_op_threshold_gpu)
SPLA_B200_CTX_SETTER(spla_ctx_set_tile_size_gpu, set_tile_size_gpu)
#undef SPLA_B200_CTX_SETTER

SplaError spla_ctx_set_alloc_host(SplaContext ctx, void* (*a)(size_t), void (*f)(void*)) {
  if (!ctx) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] {
    if (!a || !f) throw spla::InvalidAllocatorFunctionError();
    as_ctx(ctx).set_alloc_host(a, f);
  });
}
SplaError spla_ctx_set_alloc_pinned(SplaContext ctx, void* (*a)(size_t), void (*f)(void*)) {
  if (!ctx) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] {
    if (!a || !f) throw spla::InvalidAllocatorFunctionError();
    as_ctx(ctx).set_alloc_pinned(a, f);
  });
}
SplaError spla_ctx_set_alloc_gpu(SplaContext ctx, void* (*a)(size_t), void (*f)(void*)) {
  if (!ctx) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] {
    if (!a || !f) throw spla::InvalidAllocatorFunctionError();
    as_ctx(ctx).set_alloc_gpu(a, f);
  });
}

// Library extensions (no reference counterpart): select the FP64 contraction
// path of a context. path: 0 auto, 1 FP64 DMMA, 2 Ozaki INT8, 3 3xTF32 (float
// dtypes); moduli 0 = default.
SPLA_EXPORT SplaError spla_b200_ctx_set_fp64_path(SplaContext ctx, int path, int moduli) {
  if (!ctx) return SPLA_INVALID_HANDLE_ERROR;
  if (path < 0 || path > 3 || moduli < 0 || moduli > 16 || (moduli > 0 && moduli < 8))
    return SPLA_INVALID_PARAMETER_ERROR;
  return guarded([&] {
    auto& c = spla::detail::Access::ctx(as_ctx(ctx));
    c.set_fp64_path(path);
    c.set_ozaki_moduli(moduli);
  });
}

}  // extern "C"
