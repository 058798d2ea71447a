/* spla::Context (C++ interface); member functions equal the reference's
 * include/spla/context.hpp:58-196. Move-only; holds one shared_ptr to the
 * implementation, as the reference does (context.hpp:276). */
#ifndef SPLA_CONTEXT_HPP
#define SPLA_CONTEXT_HPP
#include <complex>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include "spla/config.h"
#include "spla/types.h"

namespace spla {
class ContextInternal;
namespace detail {
struct Access;
}

class SPLA_EXPORT Context {
public:
  explicit Context(SplaProcessingUnit pu);
  Context(Context&&) = default;
  Context(const Context&) = delete;
  Context& operator=(Context&&) = default;
  Context& operator=(const Context&) = delete;

  SplaProcessingUnit processing_unit() const;
  int num_tiles() const;
  int tile_size_host() const;
  int tile_size_gpu() const;
  int op_threshold_gpu() const;
  int gpu_device_id() const;
  std::uint_least64_t allocated_memory_host() const;
  std::uint_least64_t allocated_memory_pinned() const;
  std::uint_least64_t allocated_memory_gpu() const;

  void set_num_tiles(int numTiles);
  void set_tile_size_host(int tileSizeHost);
  void set_op_threshold_gpu(int opThresholdGPU);
  void set_tile_size_gpu(int tileSizeGPU);
  void set_alloc_host(std::function<void*(std::size_t)> allocateFunc,
                      std::function<void(void*)> deallocateFunc);
  void set_alloc_pinned(std::function<void*(std::size_t)> allocateFunc,
                        std::function<void(void*)> deallocateFunc);
  void set_alloc_gpu(std::function<void*(std::size_t)> allocateFunc,
                     std::function<void(void*)> deallocateFunc);

private:
  friend struct detail::Access;
  std::shared_ptr<ContextInternal> ctxInternal_;
};
}  // namespace spla
#endif
