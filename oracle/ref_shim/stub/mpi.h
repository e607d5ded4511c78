// Stand-in for <mpi.h>: the reference's public header names MPI_Comm only as
// an opaque handle type. MPI is not installed here.
#pragma once
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
