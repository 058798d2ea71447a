// spla::MatrixDistribution and the spla_mat_dis_* C ABI (reference
// include/spla/matrix_distribution.h, src/spla/matrix_distribution.cpp,
// src/spla/matrix_distribution_internal.cpp). Parameter validation follows the
// reference (matrix_distribution_internal.cpp:45-50, :78-80, :98-123): grid and
// block sizes >= 1, order in R/r/C/c, mapping entries distinct ranks of comm.
#include <set>
#include <vector>

#include "internal.hpp"
#include "spla/matrix_distribution.h"

namespace spla {

namespace {
int comm_size_of(MPI_Comm comm) {
  int size = 0;
  if (MPI_Comm_size(comm, &size) != MPI_SUCCESS) throw MPIError();
  return size;
}
}  // namespace

MatrixDistributionInternal MatrixDistributionInternal::create_blacs_block_cyclic(
    MPI_Comm comm, char order, int rows, int cols, int rb, int cb) {
  if (order != 'R' && order != 'r' && order != 'C' && order != 'c') throw InvalidParameterError();
  if (rows < 1 || cols < 1 || rb < 1 || cb < 1) throw InvalidParameterError();
  // rank of grid position (r, c) stored at mapping[r + c * rows]
  std::vector<int> mapping(static_cast<size_t>(rows) * cols);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c)
      mapping[r + static_cast<size_t>(c) * rows] =
          (order == 'R' || order == 'r') ? r * cols + c : c * rows + r;
  return create_blacs_block_cyclic_from_mapping(comm, mapping.data(), rows, cols, rb, cb);
}

MatrixDistributionInternal MatrixDistributionInternal::create_blacs_block_cyclic_from_mapping(
    MPI_Comm comm, const int* mapping, int rows, int cols, int rb, int cb) {
  if (rows < 1 || cols < 1 || rb < 1 || cb < 1) throw InvalidParameterError();
  if (!mapping) throw InvalidParameterError();
  const int size = comm_size_of(comm);
  std::set<int> seen;
  for (long i = 0; i < long(rows) * cols; ++i) {
    if (mapping[i] < 0 || mapping[i] >= size) throw InvalidParameterError();
    if (!seen.insert(mapping[i]).second) throw InvalidParameterError();
  }
  MatrixDistributionInternal d;
  d.type_ = SPLA_DIST_BLACS_BLOCK_CYCLIC;
  d.comm_ = comm;
  d.commSize_ = size;
  d.procGridRows_ = rows;
  d.procGridCols_ = cols;
  d.rowBlockSize_ = rb;
  d.colBlockSize_ = cb;
  return d;
}

MatrixDistributionInternal MatrixDistributionInternal::create_mirror(MPI_Comm comm) {
  MatrixDistributionInternal d;
  d.type_ = SPLA_DIST_MIRROR;
  d.comm_ = comm;
  d.commSize_ = comm_size_of(comm);
  d.procGridRows_ = d.commSize_;  // reference: grid rows = communicator size
  d.procGridCols_ = 1;
  d.rowBlockSize_ = 256;
  d.colBlockSize_ = 256;
  return d;
}

MatrixDistribution::MatrixDistribution(std::shared_ptr<MatrixDistributionInternal> p)
    : descInternal_(std::move(p)) {}

MatrixDistribution MatrixDistribution::create_blacs_block_cyclic(MPI_Comm comm, char order,
                                                                 int rows, int cols, int rb,
                                                                 int cb) {
  return MatrixDistribution(std::make_shared<MatrixDistributionInternal>(
      MatrixDistributionInternal::create_blacs_block_cyclic(comm, order, rows, cols, rb, cb)));
}

MatrixDistribution MatrixDistribution::create_blacs_block_cyclic_from_mapping(
    MPI_Comm comm, const int* mapping, int rows, int cols, int rb, int cb) {
  return MatrixDistribution(std::make_shared<MatrixDistributionInternal>(
      MatrixDistributionInternal::create_blacs_block_cyclic_from_mapping(comm, mapping, rows,
                                                                         cols, rb, cb)));
}

MatrixDistribution MatrixDistribution::create_mirror(MPI_Comm comm) {
  return MatrixDistribution(
      std::make_shared<MatrixDistributionInternal>(MatrixDistributionInternal::create_mirror(comm)));
}

int MatrixDistribution::proc_grid_rows() const { return descInternal_->proc_grid_rows(); }
int MatrixDistribution::proc_grid_cols() const { return descInternal_->proc_grid_cols(); }
int MatrixDistribution::row_block_size() const { return descInternal_->row_block_size(); }
int MatrixDistribution::col_block_size() const { return descInternal_->col_block_size(); }
SplaDistributionType MatrixDistribution::type() const { return descInternal_->type(); }
MPI_Comm MatrixDistribution::comm() { return descInternal_->comm(); }
void MatrixDistribution::set_row_block_size(int v) {
  if (v < 1) throw InvalidParameterError();
  descInternal_->set_row_block_size(v);
}
void MatrixDistribution::set_col_block_size(int v) {
  if (v < 1) throw InvalidParameterError();
  descInternal_->set_col_block_size(v);
}

}  // namespace spla

namespace {
template <typename F>
SplaError guarded(F&& f) {
  try {
    f();
  } catch (const spla::GenericError& e) {
    return e.error_code();
  } catch (...) {
    return SPLA_UNKNOWN_ERROR;
  }
  return SPLA_SUCCESS;
}
spla::MatrixDistribution& as_dist(SplaMatrixDistribution d) {
  return *static_cast<spla::MatrixDistribution*>(d);
}
}  // namespace

extern "C" {

SplaError spla_mat_dis_create_block_cyclic(SplaMatrixDistribution* matDis, MPI_Comm comm,
                                           char order, int rows, int cols, int rb, int cb) {
  if (!matDis) return SPLA_INVALID_POINTER_ERROR;
  return guarded([&] {
    *matDis = new spla::MatrixDistribution(
        spla::MatrixDistribution::create_blacs_block_cyclic(comm, order, rows, cols, rb, cb));
  });
}

SplaError spla_mat_dis_create_blacs_block_cyclic_from_mapping(SplaMatrixDistribution* matDis,
                                                              MPI_Comm comm, const int* mapping,
                                                              int rows, int cols, int rb, int cb) {
  if (!matDis) return SPLA_INVALID_POINTER_ERROR;
  return guarded([&] {
    *matDis = new spla::MatrixDistribution(
        spla::MatrixDistribution::create_blacs_block_cyclic_from_mapping(comm, mapping, rows, cols,
                                                                         rb, cb));
  });
}

SplaError spla_mat_dis_create_mirror(SplaMatrixDistribution* matDis, MPI_Comm comm) {
  if (!matDis) return SPLA_INVALID_POINTER_ERROR;
  return guarded([&] {
    *matDis = new spla::MatrixDistribution(spla::MatrixDistribution::create_mirror(comm));
  });
}

SplaError spla_mat_dis_destroy(SplaMatrixDistribution* matDis) {
  if (!matDis || !*matDis) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] {
    delete static_cast<spla::MatrixDistribution*>(*matDis);
    *matDis = nullptr;
  });
}

#define SPLA_B200_DIS_GETTER(NAME, TYPE, EXPR)                \
  SplaError NAME(SplaMatrixDistribution d, TYPE* out) {       \
    if (!d) return SPLA_INVALID_HANDLE_ERROR;                 \
    return guarded([&] { *out = as_dist(d).EXPR(); });        \
  }
SPLA_B200_DIS_GETTER(spla_mat_dis_proc_grid_rows, int, proc_grid_rows)
SPLA_B200_DIS_GETTER(spla_mat_dis_proc_grid_cols, int, proc_grid_cols)
SPLA_B200_DIS_GETTER(spla_mat_dis_row_block_size, int, row_block_size)
SPLA_B200_DIS_GETTER(spla_mat_dis_col_block_size, int, col_block_size)
SPLA_B200_DIS_GETTER(spla_mat_dis_type, SplaDistributionType, type)
SPLA_B200_DIS_GETTER(spla_mat_dis_comm, MPI_Comm, comm)
#undef SPLA_B200_DIS_GETTER

SplaError spla_mat_dis_set_row_block_size(SplaMatrixDistribution d, int v) {
  if (!d) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] { as_dist(d).set_row_block_size(v); });
}
SplaError spla_mat_dis_set_col_block_size(SplaMatrixDistribution d, int v) {
  if (!d) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] { as_dist(d).set_col_block_size(v); });
}

SplaError spla_mat_dis_create_block_cyclic_fortran(SplaMatrixDistribution* matDis, int commF,
                                                   char order, int rows, int cols, int rb,
                                                   int cb) {
  return spla_mat_dis_create_block_cyclic(matDis, MPI_Comm_f2c(commF), order, rows, cols, rb, cb);
}
SplaError spla_mat_dis_create_blacs_block_cyclic_from_mapping_fortran(
    SplaMatrixDistribution* matDis, int commF, const int* mapping, int rows, int cols, int rb,
    int cb) {
  return spla_mat_dis_create_blacs_block_cyclic_from_mapping(matDis, MPI_Comm_f2c(commF), mapping,
                                                             rows, cols, rb, cb);
}
SplaError spla_mat_dis_create_mirror_fortran(SplaMatrixDistribution* matDis, int commF) {
  return spla_mat_dis_create_mirror(matDis, MPI_Comm_f2c(commF));
}
SplaError spla_mat_dis_comm_fortran(SplaMatrixDistribution d, int* commF) {
  if (!d) return SPLA_INVALID_HANDLE_ERROR;
  return guarded([&] { *commF = MPI_Comm_c2f(as_dist(d).comm()); });
}

}  // extern "C"
