/*
 * Single-rank MPI stand-in for building this library on machines without an
 * MPI installation. Only what the single-rank path needs: the communicator
 * handle type, the predefined communicators and size/rank queries that answer
 * one rank. Handle values follow MPICH's integer encoding. Build against a
 * real <mpi.h> (and link libmpi) to use genuine communicators instead.
 */
#ifndef SPLA_B200_SINGLE_RANK_MPI_H
#define SPLA_B200_SINGLE_RANK_MPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Fint;

#define SPLA_B200_SINGLE_RANK_MPI 1
#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0x04000000
#define MPI_COMM_WORLD 0x44000000
#define MPI_COMM_SELF 0x44000001

static inline int MPI_Comm_size(MPI_Comm comm, int *size) {
  *size = 1;
  return comm == MPI_COMM_NULL ? 5 : MPI_SUCCESS;
}
static inline int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  *rank = 0;
  return comm == MPI_COMM_NULL ? 5 : MPI_SUCCESS;
}
static inline MPI_Comm MPI_Comm_f2c(MPI_Fint f) { return (MPI_Comm)f; }
static inline MPI_Fint MPI_Comm_c2f(MPI_Comm c) { return (MPI_Fint)c; }

#ifdef __cplusplus
}
#endif
#endif
