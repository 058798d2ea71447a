// Internal state behind spla::Context and spla::MatrixDistribution, and the
// local GEMM engine that drives the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <mpi.h>

#include <complex>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <string>

#include "spla/context.hpp"
#include "spla/exceptions.hpp"
#include "spla/matrix_distribution.hpp"
#include "spla/types.h"

namespace spla {

// Map a CUDA runtime status to the SPLA exception the reference raises for it
// (src/gpu_util/gpu_runtime_api.hpp:113-123).
void check_cuda(cudaError_t err);

// Map a splab status to an SPLA exception.
void check_splab(int status);

// One pool of memory obtained from an allocate/deallocate pair. Keeps a single
// reusable buffer per slot and grows it on demand; tracks the bytes held.
class ScratchPool {
public:
  using AllocFn = std::function<void*(std::size_t)>;
  using FreeFn = std::function<void(void*)>;
  enum Kind { kHost, kPinned, kDevice };

  ScratchPool(Kind kind, AllocFn a, FreeFn f) : kind_(kind), alloc_(std::move(a)), free_(std::move(f)) {}
  ~ScratchPool() { release(); }
  ScratchPool(const ScratchPool&) = delete;
  ScratchPool& operator=(const ScratchPool&) = delete;

  // Buffer `slot` with at least `bytes` bytes (contents not preserved on growth).
  void* get(int slot, std::size_t bytes);
  void release();
  std::uint64_t bytes_held() const { return held_; }
  void set_functions(AllocFn a, FreeFn f) {
    release();
    alloc_ = std::move(a);
    free_ = std::move(f);
  }

private:
  static constexpr int kSlots = 8;
  Kind kind_;
  AllocFn alloc_;
  FreeFn free_;
  void* ptr_[kSlots] = {nullptr};
  std::size_t size_[kSlots] = {0};
  std::uint64_t held_ = 0;
};

class ContextInternal {
public:
  explicit ContextInternal(SplaProcessingUnit pu);
  ~ContextInternal();

  SplaProcessingUnit processing_unit() const { return pu_; }
  int num_tiles() const { return numTiles_; }
  int tile_size_host() const { return tileSizeHost_; }
  int tile_size_gpu() const { return tileSizeGPU_; }
  int op_threshold_gpu() const { return opThresholdGPU_; }
  int gpu_device_id() const { return deviceId_; }

  void set_num_tiles(int v) {
    if (v < 1) throw InvalidParameterError();
    numTiles_ = v;
  }
  void set_tile_size_host(int v) {
    if (v < 1) throw InvalidParameterError();
    tileSizeHost_ = v;
  }
  void set_tile_size_gpu(int v) {
    if (v < 1) throw InvalidParameterError();
    tileSizeGPU_ = v;
  }
  void set_op_threshold_gpu(int v) {
    if (v < 0) throw InvalidParameterError();
    opThresholdGPU_ = v;
  }

  ScratchPool& host_pool() { return *host_; }
  ScratchPool& pinned_pool() { return *pinned_; }
  ScratchPool& device_pool() { return *device_; }

  // Streams and events are created lazily on the context's device.
  cudaStream_t compute_stream();
  cudaStream_t copy_stream();
  cudaEvent_t event(int i);

  // Contraction path for double / complex double: SPLAB_PATH_* (default
  // from SPLA_B200_PATH = auto | dmma | ozaki) and Ozaki modulus count.
  int fp64_path() const { return fp64Path_; }
  int ozaki_moduli() const { return ozakiModuli_; }
  void set_fp64_path(int p) { fp64Path_ = p; }
  void set_ozaki_moduli(int n) { ozakiModuli_ = n; }

private:
  SplaProcessingUnit pu_;
  int numTiles_ = 4;
  int tileSizeHost_;
  int tileSizeGPU_ = 2048;
  int opThresholdGPU_ = 2000000;
  int deviceId_ = 0;
  bool hasDevice_ = false;  // a device was present at construction
  int fp64Path_ = 0;
  int ozakiModuli_ = 0;
  std::unique_ptr<ScratchPool> host_, pinned_, device_;
  cudaStream_t compute_ = nullptr, copy_ = nullptr;
  cudaEvent_t events_[8] = {nullptr};
};

class MatrixDistributionInternal {
public:
  static MatrixDistributionInternal create_blacs_block_cyclic(MPI_Comm comm, char order,
                                                              int procGridRows, int procGridCols,
                                                              int rowBlockSize, int colBlockSize);
  static MatrixDistributionInternal create_blacs_block_cyclic_from_mapping(
      MPI_Comm comm, const int* mapping, int procGridRows, int procGridCols, int rowBlockSize,
      int colBlockSize);
  static MatrixDistributionInternal create_mirror(MPI_Comm comm);

  int proc_grid_rows() const { return procGridRows_; }
  int proc_grid_cols() const { return procGridCols_; }
  int row_block_size() const { return rowBlockSize_; }
  int col_block_size() const { return colBlockSize_; }
  SplaDistributionType type() const { return type_; }
  MPI_Comm comm() const { return comm_; }
  int comm_size() const { return commSize_; }
  void set_row_block_size(int v) { rowBlockSize_ = v; }
  void set_col_block_size(int v) { colBlockSize_ = v; }

private:
  MatrixDistributionInternal() = default;
  SplaDistributionType type_ = SPLA_DIST_MIRROR;
  MPI_Comm comm_ = MPI_COMM_SELF;
  int commSize_ = 1;
  int procGridRows_ = 1, procGridCols_ = 1;
  int rowBlockSize_ = 256, colBlockSize_ = 256;
};

namespace detail {
// Access to the implementation objects of the public classes.
struct Access {
  static ContextInternal& ctx(Context& c) { return *c.ctxInternal_; }
  static const ContextInternal& ctx(const Context& c) { return *c.ctxInternal_; }
  static MatrixDistributionInternal& dist(MatrixDistribution& d) { return *d.descInternal_; }
  static MatrixDistribution make_dist(std::shared_ptr<MatrixDistributionInternal> p) {
    return MatrixDistribution(std::move(p));
  }
};
}  // namespace detail

// The local GEMM engine (reference src/gemm/gemm_gpu.cpp:59-174 and
// src/gpu_util/multiply_gpu.cpp:78-143): C <- alpha*op(A)*op(B) + beta*C with
// any mix of host and device pointers, computed on the context's GPU.
// `check_order_host` selects nothing here; validation happens in the callers.
template <typename T>
void local_gemm(ContextInternal& ctx, SplaOperation opA, SplaOperation opB, int m, int n, int k,
                T alpha, const T* A, int lda, const T* B, int ldb, T beta, T* C, int ldc,
                SplaFillMode fill = SPLA_FILL_MODE_FULL, int ro = 0, int co = 0);

}  // namespace spla
