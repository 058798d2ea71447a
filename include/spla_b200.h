/* Extensions of this library beyond the SPLA interface (no reference
 * counterpart). Declared separately so that include/spla/ stays identical in
 * content to the interface it replaces. */
#ifndef SPLA_B200_H
#define SPLA_B200_H
#include "spla/context.h"
#include "spla/errors.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Select the contraction path a context uses (all dtypes): path 0 =
 * automatic, 1 = FP64 tensor cores (DMMA; float inputs accumulate in FP64),
 * 2 = Ozaki scheme II on INT8 tensor cores, 3 = 3xTF32 tensor cores (float and
 * complex float ssb-shaped problems; double problems use DMMA). moduli =
 * number of CRT moduli for path 2 (0 = default: 15 for double, <= 1e-14
 * relative error; 9 for float); valid: 0 or 8..16. The environment variables
 * SPLA_B200_PATH (auto|dmma|ozaki|tf32x3) and SPLA_B200_OZAKI_MODULI set the
 * defaults of new contexts. */
SPLA_EXPORT SplaError spla_b200_ctx_set_fp64_path(SplaContext ctx, int path, int moduli);

#ifdef __cplusplus
}
#endif
#endif
