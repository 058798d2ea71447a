/* Enumerations of the SPLA interface. Values and order are part of the ABI and
 * equal the reference's (include/spla/types.h:33-83). */
#ifndef SPLA_TYPES_H
#define SPLA_TYPES_H
#include "spla/config.h"

/* How a matrix is laid out over the ranks of a communicator. */
enum SplaDistributionType {
  SPLA_DIST_BLACS_BLOCK_CYCLIC, /* ScaLAPACK-style 2D block-cyclic */
  SPLA_DIST_MIRROR              /* every rank holds the whole matrix */
};

/* Where a Context computes. Both run on the GPU in this library: a HOST context
 * keeps host-side validation order and expects host-resident operands. */
enum SplaProcessingUnit { SPLA_PU_HOST, SPLA_PU_GPU };

/* op() applied to an operand. */
enum SplaOperation { SPLA_OP_NONE, SPLA_OP_TRANSPOSE, SPLA_OP_CONJ_TRANSPOSE };

/* Part of C that pgemm_ssbtr must produce. */
enum SplaFillMode { SPLA_FILL_MODE_FULL, SPLA_FILL_MODE_UPPER, SPLA_FILL_MODE_LOWER };

#ifndef __cplusplus
typedef enum SplaDistributionType SplaDistributionType;
typedef enum SplaProcessingUnit SplaProcessingUnit;
typedef enum SplaOperation SplaOperation;
typedef enum SplaFillMode SplaFillMode;
#endif
#endif
