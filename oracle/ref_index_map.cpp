// Test infrastructure: a C-callable window onto the reference's own block-cyclic
// index map and fill-mode predicate, compiled from the reference sources into
// oracle/_ref/libspla_ref.so. Used only by the index-map parity tests.
#include "block_generation/block.hpp"
#include "block_generation/block_cyclic_generator.hpp"

extern "C" {

long ref_num_blocks(long rb, long cb, long gr, long gc, long nr, long nc, long ro, long co) {
  spla::BlockCyclicGenerator gen(rb, cb, gr, gc, nr, nc, ro, co);
  return gen.num_blocks();
}

void ref_block_info(long rb, long cb, long gr, long gc, long nr, long nc, long ro, long co,
                    long blockIdx, long *out) {
  spla::BlockCyclicGenerator gen(rb, cb, gr, gc, nr, nc, ro, co);
  const spla::BlockInfo b = gen.get_block_info(blockIdx);
  out[0] = b.globalRowIdx;
  out[1] = b.globalColIdx;
  out[2] = b.globalSubRowIdx;
  out[3] = b.globalSubColIdx;
  out[4] = b.localRowIdx;
  out[5] = b.localColIdx;
  out[6] = b.numRows;
  out[7] = b.numCols;
  out[8] = b.mpiRank;
}

long ref_local_rows(long rb, long cb, long gr, long gc, long nr, long nc, long ro, long co,
                    long rank) {
  spla::BlockCyclicGenerator gen(rb, cb, gr, gc, nr, nc, ro, co);
  return gen.local_rows(rank);
}

long ref_local_cols(long rb, long cb, long gr, long gc, long nr, long nc, long ro, long co,
                    long rank) {
  spla::BlockCyclicGenerator gen(rb, cb, gr, gc, nr, nc, ro, co);
  return gen.local_cols(rank);
}

int ref_block_is_active(long row, long col, long numRows, long numCols, long ro, long co,
                        int mode) {
  spla::Block b{row, col, numRows, numCols};
  return spla::block_is_active(b, ro, co, static_cast<SplaFillMode>(mode)) ? 1 : 0;
}
}
