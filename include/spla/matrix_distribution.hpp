/* spla::MatrixDistribution (C++ interface); member functions equal the
 * reference's include/spla/matrix_distribution.hpp:60-84. Copyable; holds one
 * shared_ptr to the implementation (matrix_distribution.hpp:220). */
#ifndef SPLA_MATRIX_DISTRIBUTION_HPP
#define SPLA_MATRIX_DISTRIBUTION_HPP
#include <mpi.h>
#include <complex>
#include <memory>
#include "spla/config.h"
#include "spla/types.h"

namespace spla {
class MatrixDistributionInternal;
class Context;
namespace detail {
struct Access;
}

class SPLA_EXPORT MatrixDistribution {
public:
  static MatrixDistribution create_blacs_block_cyclic(MPI_Comm comm, char order, int procGridRows,
                                                      int procGridCols, int rowBlockSize,
                                                      int colBlockSize);
  static MatrixDistribution create_blacs_block_cyclic_from_mapping(
      MPI_Comm comm, const int* mapping, int procGridRows, int procGridCols, int rowBlockSize,
      int colBlockSize);
  static MatrixDistribution create_mirror(MPI_Comm comm);

  MatrixDistribution(MatrixDistribution&&) = default;
  MatrixDistribution(const MatrixDistribution&) = default;
  MatrixDistribution& operator=(MatrixDistribution&&) = default;
  MatrixDistribution& operator=(const MatrixDistribution&) = default;

  int proc_grid_rows() const;
  int proc_grid_cols() const;
  int row_block_size() const;
  int col_block_size() const;
  SplaDistributionType type() const;
  MPI_Comm comm();
  void set_row_block_size(int rowBlockSize);
  void set_col_block_size(int colBlockSize);

private:
  friend struct detail::Access;
  explicit MatrixDistribution(std::shared_ptr<MatrixDistributionInternal> descInternal);
  std::shared_ptr<MatrixDistributionInternal> descInternal_;
};
}  // namespace spla
#endif
