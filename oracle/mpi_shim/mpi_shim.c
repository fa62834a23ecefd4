/*
 * Single-rank MPI stand-in (see mpi.h). TEST INFRASTRUCTURE only.
 *
 * MPI_Abort does not end the process: it records the error code so that
 * a test driving the reference's NaN-abort path
 * (src/physics/src/physics_runge_kutta_interface.c:352-355) can observe it.
 */
#include "mpi.h"

#include <stdio.h>
#include <string.h>
#include <time.h>

static int g_abort_code = 0;

static size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_INT:        return sizeof(int);
    case MPI_DOUBLE:     return sizeof(double);
    case MPI_DOUBLE_INT: return sizeof(double) + sizeof(int) + 4; /* padded struct */
    default:             return 0;
    }
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1.0e-9 * (double)ts.tv_nsec;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)op; (void)comm;
    memmove(recvbuf, sendbuf, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count,
               MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm)
{
    (void)root;
    return MPI_Allreduce(sendbuf, recvbuf, count, type, op, comm);
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *request)
{
    (void)buf; (void)count; (void)type; (void)source; (void)tag; (void)comm;
    *request = 0;
    return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *request)
{
    (void)buf; (void)count; (void)type; (void)dest; (void)tag; (void)comm;
    *request = 0;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *requests, MPI_Status *statuses)
{
    (void)count; (void)requests; (void)statuses;
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm comm, int errorcode)
{
    (void)comm;
    g_abort_code = errorcode;
    fprintf(stderr, "[mpi shim] MPI_Abort(%d)\n", errorcode);
    return MPI_SUCCESS;
}

/* Error code of the last MPI_Abort, 0 if none; cleared by the read. */
int oracle_mpi_take_abort_code(void)
{
    int c = g_abort_code;
    g_abort_code = 0;
    return c;
}
