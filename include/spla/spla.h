/* Umbrella header of the C interface (same set as the reference's include/spla/spla.h:31-40;
 * pgemm_ssbtr.h is included directly by users, as with the reference). */
#ifndef SPLA_SPLA_H
#define SPLA_SPLA_H
#include <mpi.h>
#include "spla/config.h"
#include "spla/context.h"
#include "spla/matrix_distribution.h"
#include "spla/pgemm_sbs.h"
#include "spla/pgemm_ssb.h"
#include "spla/gemm.h"
#include "spla/errors.h"
#include "spla/types.h"
#endif
