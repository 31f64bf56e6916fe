/* Single-rank MPI stand-in used only to compile the reference's own headers (include/darray.h and friends)
 * for oracle pinning.  Every collective at world size 1 is a local copy; point-to-point calls between
 * distinct ranks cannot occur and abort.  MPI_BYTE counts bytes, as real MPI does (the reference passes
 * element counts with MPI_BYTE for non-float types, include/darray.h:55-63; that is reproduced, not fixed). */
#pragma once
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_FLOAT_INT 5
#define MPI_SUM 0
#define MPI_MAXLOC 1

static inline size_t mpistub_size(MPI_Datatype t) {
  switch (t) {
    case MPI_BYTE: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_FLOAT_INT: return sizeof(float) + sizeof(int);
  }
  return 1;
}
static inline void mpistub_copy(void* dst, const void* src, int count, MPI_Datatype t) {
  if (count > 0 && dst != src) memmove(dst, src, (size_t)count * mpistub_size(t));
}
static inline void mpistub_unreachable(const char* what) {
  fprintf(stderr, "mpi stub: %s between distinct ranks cannot happen at world size 1\n", what);
  abort();
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  mpistub_copy(r, s, n, t); return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
  mpistub_copy(r, s, sn, st); return MPI_SUCCESS;
}
static inline int MPI_Allgatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs,
                                 MPI_Datatype rt, MPI_Comm) {
  mpistub_copy((char*)r + (size_t)displs[0] * mpistub_size(rt), s, sn, st); return MPI_SUCCESS;
}
static inline int MPI_Sendrecv(const void* s, int sn, MPI_Datatype st, int, int, void* r, int, MPI_Datatype, int,
                               int, MPI_Comm, MPI_Status*) {
  mpistub_copy(r, s, sn, st); return MPI_SUCCESS;
}
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int*,
                                const int* rd, MPI_Datatype rt, MPI_Comm) {
  mpistub_copy((char*)r + (size_t)rd[0] * mpistub_size(rt), (const char*)s + (size_t)sd[0] * mpistub_size(st), sc[0],
               st);
  return MPI_SUCCESS;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { mpistub_unreachable("MPI_Send"); return 1; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { mpistub_unreachable("MPI_Recv"); return 1; }
