/* Umbrella header of the C++ interface (same set as the reference's include/spla/spla.hpp:36-42). */
#ifndef SPLA_SPLA_HPP
#define SPLA_SPLA_HPP
#include "spla/config.h"
#include "spla/context.hpp"
#include "spla/exceptions.hpp"
#include "spla/gemm.hpp"
#include "spla/matrix_distribution.hpp"
#include "spla/pgemm_sbs.hpp"
#include "spla/pgemm_ssb.hpp"
#include "spla/types.h"
#endif
