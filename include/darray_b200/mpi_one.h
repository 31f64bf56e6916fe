// Single-process stand-ins for the few MPI calls the reference's drivers make around DArray
// (MPI_Init, MPI_Comm_size, ...), so that one-rank code builds without an MPI installation.  Define
// DARRAY_B200_HAVE_MPI to use a real <mpi.h> instead (at world size 1).
#pragma once
#ifdef DARRAY_B200_HAVE_MPI
#include <mpi.h>
#else
typedef int MPI_Comm;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif
#ifndef MPI_SUCCESS
#define MPI_SUCCESS 0
#endif
inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
#endif
