/*
 * Oracle-only single-process stand-in for the MPI symbols the reference's serial 2D path
 * touches: instrumentor/timer.h:36-40, instrumentor/profiler.h:67-71 and
 * base/parallel/mpi/mpi_misc.cpp:27-50. With no MPI launcher the reference never calls them
 * (MPIUtils::is_mpi() is false), but they must compile. TEST INFRASTRUCTURE only.
 */
#pragma once

typedef int MPI_Comm;
typedef int MPI_Datatype;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_SUCCESS 0

static inline int MPI_Comm_rank(MPI_Comm, int* rank)
{
    *rank = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm, int* size)
{
    *size = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
