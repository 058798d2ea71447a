/* Build configuration for compiling the unmodified reference host library
 * as the oracle (host BLAS through the CBLAS interface, no GPU backend).
 * Replaces the CMake-generated include/spla/config.h (reference
 * include/spla/config.h.in:33-44). Test infrastructure only. */
#ifndef SPLA_CONFIG_H
#define SPLA_CONFIG_H
#define SPLA_CBLAS
#define SPLA_RESTRICT_ATTR __restrict__
#include "spla/spla_export.h"
#endif
