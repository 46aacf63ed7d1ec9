/*
 * Single-rank stand-in for <mpi.h>, used ONLY to compile the reference
 * BioFVM/DistPhy sources into the CPU oracle (test infrastructure).
 *
 * The world has exactly one rank (rank 0, size 1).  With one rank the
 * reference LOD solver (BioFVM/BioFVM_solvers.cpp:102-780) executes no
 * point-to-point call: only MPI_Barrier, which is a no-op here.  Every call
 * that would move data between ranks aborts loudly, so a code path that
 * needs a second rank can never silently produce a single-rank answer.
 *
 * Written for this project; it is not derived from any MPI implementation.
 */
#ifndef BFVM_ORACLE_MPI_SHIM_H
#define BFVM_ORACLE_MPI_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct { int fd; } MPI_File;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count_;
} MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-1)

#define MPI_CHAR 1
#define MPI_CHARACTER 1
#define MPI_INT 2
#define MPI_UNSIGNED 3
#define MPI_DOUBLE 4
#define MPI_PACKED 5
#define MPI_BYTE 6

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

#define MPI_MODE_WRONLY 1
#define MPI_MODE_CREATE 2

#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

static inline int bfvm_shim_abort_(const char* what) {
  fprintf(stderr, "oracle mpi shim: %s needs more than one rank; aborting\n", what);
  abort();
  return 1;
}

static inline int MPI_Init_thread(int*, char***, int required, int* provided) {
  *provided = required;
  return MPI_SUCCESS;
}
static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int, MPI_Comm* out) {
  *out = MPI_COMM_WORLD;
  return MPI_SUCCESS;
}
static inline int MPI_Cart_coords(MPI_Comm, int, int ndims, int* coords) {
  for (int i = 0; i < ndims; ++i) coords[i] = 0;
  return MPI_SUCCESS;
}
static inline int MPI_Cart_shift(MPI_Comm, int, int, int* src, int* dst) {
  *src = MPI_PROC_NULL;
  *dst = MPI_PROC_NULL;
  return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) {
  fprintf(stderr, "oracle mpi shim: MPI_Abort(%d)\n", code);
  abort();
  return 1;
}

/* Data movement between ranks: never legal with one rank. */
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return bfvm_shim_abort_("MPI_Isend"); }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return bfvm_shim_abort_("MPI_Irecv"); }
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return bfvm_shim_abort_("MPI_Send"); }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return bfvm_shim_abort_("MPI_Recv"); }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return bfvm_shim_abort_("MPI_Wait"); }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return bfvm_shim_abort_("MPI_Waitall"); }
static inline int MPI_Get_count(const MPI_Status*, MPI_Datatype, int*) { return bfvm_shim_abort_("MPI_Get_count"); }
static inline int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return bfvm_shim_abort_("MPI_Allreduce"); }
static inline int MPI_Reduce(const void*, void*, int, MPI_Datatype, MPI_Op, int, MPI_Comm) { return bfvm_shim_abort_("MPI_Reduce"); }
static inline int MPI_Allgather(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm) { return bfvm_shim_abort_("MPI_Allgather"); }
static inline int MPI_Gather(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, int, MPI_Comm) { return bfvm_shim_abort_("MPI_Gather"); }
static inline int MPI_Scatter(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, int, MPI_Comm) { return bfvm_shim_abort_("MPI_Scatter"); }

/* MPI-IO (density output through MPI files): not part of the oracle. */
static inline int MPI_File_open(MPI_Comm, const char*, int, MPI_Info, MPI_File*) { return bfvm_shim_abort_("MPI_File_open"); }
static inline int MPI_File_close(MPI_File*) { return bfvm_shim_abort_("MPI_File_close"); }
static inline int MPI_File_write(MPI_File, const void*, int, MPI_Datatype, MPI_Status*) { return bfvm_shim_abort_("MPI_File_write"); }
static inline int MPI_File_get_size(MPI_File, MPI_Offset*) { return bfvm_shim_abort_("MPI_File_get_size"); }
static inline int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char*, MPI_Info) { return bfvm_shim_abort_("MPI_File_set_view"); }

#endif
