/*
 * Single-rank MPI stand-in used ONLY to compile the unmodified reference host
 * library (SPLA's src/) into oracle/_ref/libspla_ref.so. Test infrastructure:
 * nothing in the product includes this header.
 *
 * Every communicator has exactly one rank. Communicator management, groups
 * and derived datatypes are accepted as no-ops; point-to-point and collective
 * calls are unreachable at communicator size 1 (the reference short-circuits
 * to a local GEMM: src/pgemm_ssb/pgemm_ssb_host.cpp:168-171,
 * src/pgemm_sbs/pgemm_sbs_host.cpp:179-183) and abort if reached.
 *
 * MPI_Comm is an int with MPICH-compatible handle values so that the same
 * integer can be passed to both this library and the product library
 * (whose own single-rank stand-in uses the same values).
 */
#ifndef ORACLE_SINGLE_RANK_MPI_H
#define ORACLE_SINGLE_RANK_MPI_H

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Group;
typedef int MPI_Request;
typedef int MPI_Win;
typedef int MPI_Info;
typedef int MPI_Op;
typedef int MPI_Fint;
typedef ptrdiff_t MPI_Aint;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_NULL 0x04000000
#define MPI_COMM_WORLD 0x44000000
#define MPI_COMM_SELF 0x44000001
#define MPI_GROUP_EMPTY 0x48000000
#define MPI_DATATYPE_NULL 0x0c000000
#define MPI_REQUEST_NULL 0x2c000000
#define MPI_INFO_NULL 0x1c000000
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)-1)
#define MPI_SUM 0x58000003
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_COMBINER_NAMED 1
#define MPI_COMBINER_DUP 2
#define MPI_ORDER_FORTRAN 57

#define MPI_CHAR 0x4c000101
#define MPI_SIGNED_CHAR 0x4c000118
#define MPI_UNSIGNED_CHAR 0x4c000102
#define MPI_SHORT 0x4c000203
#define MPI_UNSIGNED_SHORT 0x4c000204
#define MPI_INT 0x4c000405
#define MPI_UNSIGNED 0x4c000406
#define MPI_LONG 0x4c000807
#define MPI_UNSIGNED_LONG 0x4c000808
#define MPI_LONG_LONG 0x4c000809
#define MPI_UNSIGNED_LONG_LONG 0x4c000819
#define MPI_FLOAT 0x4c00040a
#define MPI_DOUBLE 0x4c00080b
#define MPI_LONG_DOUBLE 0x4c00100c
#define MPI_C_BOOL 0x4c00013f
#define MPI_COMPLEX 0x4c00081e
#define MPI_DOUBLE_COMPLEX 0x4c001022
#define MPI_CXX_FLOAT_COMPLEX 0x4c000834
#define MPI_CXX_DOUBLE_COMPLEX 0x4c001035
#define MPI_C_FLOAT_COMPLEX 0x4c000840
#define MPI_C_DOUBLE_COMPLEX 0x4c001041

static inline int oracle_mpi_unreachable(const char *what) {
  fprintf(stderr, "single-rank MPI stand-in: %s is unreachable at communicator size 1\n", what);
  abort();
  return MPI_ERR_OTHER;
}

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Init_thread(int *, char ***, int, int *provided) {
  *provided = MPI_THREAD_MULTIPLE;
  return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int *flag) { *flag = 0; return MPI_SUCCESS; }
static inline int MPI_Finalized(int *flag) { *flag = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *out) { *out = comm; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group *group) { *group = 1; return MPI_SUCCESS; }
static inline int MPI_Group_incl(MPI_Group, int, const int *, MPI_Group *out) {
  *out = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Group_free(MPI_Group *group) { *group = MPI_GROUP_EMPTY; return MPI_SUCCESS; }
static inline int MPI_Comm_create_group(MPI_Comm comm, MPI_Group, int, MPI_Comm *out) {
  *out = comm;
  return MPI_SUCCESS;
}
static inline MPI_Comm MPI_Comm_f2c(MPI_Fint f) { return (MPI_Comm)f; }
static inline MPI_Fint MPI_Comm_c2f(MPI_Comm c) { return (MPI_Fint)c; }
static inline int MPI_Alloc_mem(MPI_Aint size, MPI_Info, void *baseptr) {
  void *p = malloc(size > 0 ? (size_t)size : 1);
  *(void **)baseptr = p;
  return p ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_Free_mem(void *p) { free(p); return MPI_SUCCESS; }

static inline int MPI_Type_vector(int, int, int, MPI_Datatype, MPI_Datatype *t) {
  *t = MPI_DATATYPE_NULL + 1;
  return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype *t) {
  *t = MPI_DATATYPE_NULL + 1;
  return MPI_SUCCESS;
}
static inline int MPI_Type_create_hindexed(int, const int *, const MPI_Aint *, MPI_Datatype,
                                           MPI_Datatype *t) {
  *t = MPI_DATATYPE_NULL + 1;
  return MPI_SUCCESS;
}
static inline int MPI_Type_create_subarray(int, const int *, const int *, const int *, int,
                                           MPI_Datatype, MPI_Datatype *t) {
  *t = MPI_DATATYPE_NULL + 1;
  return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype *t) { *t = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
static inline int MPI_Type_get_envelope(MPI_Datatype, int *ni, int *na, int *nd, int *combiner) {
  *ni = 0; *na = 0; *nd = 0; *combiner = MPI_COMBINER_NAMED;
  return MPI_SUCCESS;
}

static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
  return oracle_mpi_unreachable("MPI_Send");
}
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  return oracle_mpi_unreachable("MPI_Isend");
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  return oracle_mpi_unreachable("MPI_Irecv");
}
static inline int MPI_Wait(MPI_Request *r, MPI_Status *) { *r = MPI_REQUEST_NULL; return MPI_SUCCESS; }
static inline int MPI_Test(MPI_Request *r, int *flag, MPI_Status *) {
  *r = MPI_REQUEST_NULL;
  *flag = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) {
  return oracle_mpi_unreachable("MPI_Bcast");
}
static inline int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) {
  return oracle_mpi_unreachable("MPI_Allreduce");
}
static inline int MPI_Iallreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm,
                                 MPI_Request *) {
  return oracle_mpi_unreachable("MPI_Iallreduce");
}
static inline int MPI_Win_create(void *, MPI_Aint, int, MPI_Info, MPI_Comm, MPI_Win *) {
  return oracle_mpi_unreachable("MPI_Win_create");
}
static inline int MPI_Win_free(MPI_Win *) { return MPI_SUCCESS; }

#ifdef __cplusplus
}
#endif

#endif
