/* Context: per-device settings, scratch memory and streams shared by calls.
 * C interface; each function replaces the reference declaration cited beside it
 * (include/spla/context.h). A Context must not be used by two threads at once. */
#ifndef SPLA_CONTEXT_H
#define SPLA_CONTEXT_H
#include <stddef.h>
#include <stdint.h>
#include "spla/config.h"
#include "spla/errors.h"
#include "spla/types.h"

typedef void* SplaContext;

#ifdef __cplusplus
extern "C" {
#endif

/* context.h:54 - create; the GPU is the current CUDA device at creation time. */
SPLA_EXPORT SplaError spla_ctx_create(SplaContext* ctx, SplaProcessingUnit pu);
/* context.h:62 - destroy and set *ctx to NULL. */
SPLA_EXPORT SplaError spla_ctx_destroy(SplaContext* ctx);
/* context.h:70 - declared but never defined by the reference; defined here. */
SPLA_EXPORT SplaError spla_ctx_processing_unit(SplaContext ctx, SplaProcessingUnit* pu);
/* context.h:78 - number of concurrent tiles (streams) for host-resident operands. */
SPLA_EXPORT SplaError spla_ctx_num_tiles(SplaContext ctx, int* numTiles);
/* context.h:86 */
SPLA_EXPORT SplaError spla_ctx_tile_size_host(SplaContext ctx, int* tileSizeHost);
/* context.h:94 - edge of the square staging tile for host-resident operands. */
SPLA_EXPORT SplaError spla_ctx_tile_size_gpu(SplaContext ctx, int* tileSizeGPU);
/* context.h:103 */
SPLA_EXPORT SplaError spla_ctx_op_threshold_gpu(SplaContext ctx, int* opThresholdGPU);
/* context.h:112 */
SPLA_EXPORT SplaError spla_ctx_gpu_device_id(SplaContext ctx, int* deviceId);
/* context.h:121 */
SPLA_EXPORT SplaError spla_ctx_allocated_memory_host(SplaContext ctx, uint_least64_t* size);
/* context.h:130 - returns the pinned pool size (the reference returns the host size). */
SPLA_EXPORT SplaError spla_ctx_allocated_memory_pinned(SplaContext ctx, uint_least64_t* size);
/* context.h:140 - returns the device pool size (the reference returns the host size). */
SPLA_EXPORT SplaError spla_ctx_allocated_memory_gpu(SplaContext ctx, uint_least64_t* size);
/* context.h:149 */
SPLA_EXPORT SplaError spla_ctx_set_num_tiles(SplaContext ctx, int numTiles);
/* context.h:158 */
SPLA_EXPORT SplaError spla_ctx_set_tile_size_host(SplaContext ctx, int tileSizeHost);
/* context.h:168 */
SPLA_EXPORT SplaError spla_ctx_set_op_threshold_gpu(SplaContext ctx, int opThresholdGPU);
/* context.h:177 */
SPLA_EXPORT SplaError spla_ctx_set_tile_size_gpu(SplaContext ctx, int tileSizeGPU);
/* context.h:188 - allocator for host scratch. */
SPLA_EXPORT SplaError spla_ctx_set_alloc_host(SplaContext ctx, void* (*allocateFunc)(size_t),
                                              void (*deallocateFunc)(void*));
/* context.h:200 - allocator for page-locked host scratch (staging buffers). */
SPLA_EXPORT SplaError spla_ctx_set_alloc_pinned(SplaContext ctx, void* (*allocateFunc)(size_t),
                                                void (*deallocateFunc)(void*));
/* context.h:212 - allocator for device scratch (split-K partials, Ozaki slices). */
SPLA_EXPORT SplaError spla_ctx_set_alloc_gpu(SplaContext ctx, void* (*allocateFunc)(size_t),
                                             void (*deallocateFunc)(void*));

#ifdef __cplusplus
}
#endif
#endif
