/*
 * mpi.h - a single-rank stand-in for the MPI calls GPUPRM's planner makes
 * (prm/src/lib/prm/prmsolver.cpp, prm/src/main.cpp), so that PRMSolver can
 * be compiled and run in one process without an MPI installation.
 *
 * TEST INFRASTRUCTURE ONLY: used by oracle/prm_dropin.cpp to run the
 * reference's planner unchanged, once with the reference's CPU checker and
 * once with the B200 checker behind the Configspace<ndof> interface.
 *
 * Semantics for a communicator of size 1: rank 0; broadcasts, barriers and
 * waits do nothing; gathers and reductions copy the caller's buffer to the
 * receive buffer (at displacement displs[0] where given).  Point-to-point
 * calls only occur with more than one rank and abort.
 */
#ifndef GPRM_MPI_SINGLE_H
#define GPRM_MPI_SINGLE_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;   /* element size in bytes */
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_FLOAT ((MPI_Datatype)sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_SUCCESS 0

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }

static inline int gprm_mpi_copy(const void* s, void* r, int count, MPI_Datatype t)
{
    if (r && s && count > 0) memmove(r, s, (size_t)count * (size_t)t);
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm)
{
    return gprm_mpi_copy(s, r, sc, st);
}
static inline int MPI_Iallgather(const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt,
                                 MPI_Comm c, MPI_Request*)
{
    return MPI_Allgather(s, sc, st, r, rc, rt, c);
}
static inline int MPI_Allgatherv(const void* s, int sc, MPI_Datatype st, void* r, const int*, const int* displs,
                                 MPI_Datatype rt, MPI_Comm)
{
    return gprm_mpi_copy(s, r ? (char*)r + (size_t)displs[0] * (size_t)rt : r, sc, st);
}
static inline int MPI_Iallgatherv(const void* s, int sc, MPI_Datatype st, void* r, const int* rc, const int* displs,
                                  MPI_Datatype rt, MPI_Comm c, MPI_Request*)
{
    return MPI_Allgatherv(s, sc, st, r, rc, displs, rt, c);
}
static inline int MPI_Gather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm)
{
    return gprm_mpi_copy(s, r, sc, st);
}
static inline int MPI_Gatherv(const void* s, int sc, MPI_Datatype st, void* r, const int*, const int* displs,
                              MPI_Datatype rt, int, MPI_Comm)
{
    return gprm_mpi_copy(s, r ? (char*)r + (size_t)(displs ? displs[0] : 0) * (size_t)rt : r, sc, st);
}
static inline int MPI_Reduce(const void* s, void* r, int c, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    return gprm_mpi_copy(s, r, c, t);
}
static inline int MPI_Allreduce(const void* s, void* r, int c, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    return gprm_mpi_copy(s, r, c, t);
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm)
{
    fprintf(stderr, "MPI_Send called with one rank\n");
    abort();
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*)
{
    fprintf(stderr, "MPI_Recv called with one rank\n");
    abort();
}

#endif
