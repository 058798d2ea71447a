/* Matrix distribution descriptors (C interface), replacing the reference
 * declarations cited beside each function (include/spla/matrix_distribution.h). */
#ifndef SPLA_MATRIX_DISTRIBUTION_H
#define SPLA_MATRIX_DISTRIBUTION_H
#include <mpi.h>
#include "spla/config.h"
#include "spla/errors.h"
#include "spla/types.h"

typedef void* SplaMatrixDistribution;

#ifdef __cplusplus
extern "C" {
#endif

/* matrix_distribution.h:59 - order 'R'/'r' (row-major rank grid) or 'C'/'c'. */
SPLA_EXPORT SplaError spla_mat_dis_create_block_cyclic(SplaMatrixDistribution* matDis,
                                                       MPI_Comm comm, char order, int procGridRows,
                                                       int procGridCols, int rowBlockSize,
                                                       int colBlockSize);
/* matrix_distribution.h:77 - mapping[r + c*procGridRows] is the rank at grid (r, c). */
SPLA_EXPORT SplaError spla_mat_dis_create_blacs_block_cyclic_from_mapping(
    SplaMatrixDistribution* matDis, MPI_Comm comm, const int* mapping, int procGridRows,
    int procGridCols, int rowBlockSize, int colBlockSize);
/* matrix_distribution.h:87 */
SPLA_EXPORT SplaError spla_mat_dis_destroy(SplaMatrixDistribution* matDis);
/* matrix_distribution.h:96 */
SPLA_EXPORT SplaError spla_mat_dis_create_mirror(SplaMatrixDistribution* matDis, MPI_Comm comm);
/* matrix_distribution.h:105 */
SPLA_EXPORT SplaError spla_mat_dis_proc_grid_rows(SplaMatrixDistribution matDis, int* procGridRows);
/* matrix_distribution.h:114 */
SPLA_EXPORT SplaError spla_mat_dis_proc_grid_cols(SplaMatrixDistribution matDis, int* procGridCols);
/* matrix_distribution.h:123 */
SPLA_EXPORT SplaError spla_mat_dis_row_block_size(SplaMatrixDistribution matDis, int* rowBlockSize);
/* matrix_distribution.h:132 */
SPLA_EXPORT SplaError spla_mat_dis_col_block_size(SplaMatrixDistribution matDis, int* colBlockSize);
/* matrix_distribution.h:141 */
SPLA_EXPORT SplaError spla_mat_dis_type(SplaMatrixDistribution matDis, SplaDistributionType* type);
/* matrix_distribution.h:151 */
SPLA_EXPORT SplaError spla_mat_dis_comm(SplaMatrixDistribution matDis, MPI_Comm* comm);
/* matrix_distribution.h:161 */
SPLA_EXPORT SplaError spla_mat_dis_set_row_block_size(SplaMatrixDistribution matDis, int rowBlockSize);
/* matrix_distribution.h:171 */
SPLA_EXPORT SplaError spla_mat_dis_set_col_block_size(SplaMatrixDistribution matDis, int colBlockSize);

/* Fortran-handle variants used by the reference's Fortran module
 * (src/spla/matrix_distribution.cpp:103-110, :128-135, :163-168, :257-260). */
SPLA_EXPORT SplaError spla_mat_dis_create_block_cyclic_fortran(SplaMatrixDistribution* matDis,
                                                               int commFortran, char order,
                                                               int procGridRows, int procGridCols,
                                                               int rowBlockSize, int colBlockSize);
SPLA_EXPORT SplaError spla_mat_dis_create_blacs_block_cyclic_from_mapping_fortran(
    SplaMatrixDistribution* matDis, int commFortran, const int* mapping, int procGridRows,
    int procGridCols, int rowBlockSize, int colBlockSize);
SPLA_EXPORT SplaError spla_mat_dis_create_mirror_fortran(SplaMatrixDistribution* matDis,
                                                         int commFortran);
SPLA_EXPORT SplaError spla_mat_dis_comm_fortran(SplaMatrixDistribution matDis, int* commFortran);

#ifdef __cplusplus
}
#endif
#endif
