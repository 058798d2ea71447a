/* Build configuration of the B200 implementation of the SPLA interface.
 * Counterpart of the reference's generated config (include/spla/config.h.in:33-44).
 * SPLA_CUDA is always set: this library computes on an NVIDIA B200 (sm_100a). */
#ifndef SPLA_CONFIG_H
#define SPLA_CONFIG_H
#define SPLA_CUDA
#define SPLA_RESTRICT_ATTR __restrict__
#ifndef SPLA_EXPORT
#define SPLA_EXPORT __attribute__((visibility("default")))
#endif
#endif
