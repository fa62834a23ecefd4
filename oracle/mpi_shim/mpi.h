/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's
 * own C physics driver (src/physics/src/*.c) into the CPU oracle library.
 *
 * TEST INFRASTRUCTURE: nothing in the product links against this file.
 *
 * Every call behaves as it would on an MPI_COMM_WORLD of size 1:
 * reductions copy the send buffer, point-to-point calls are only reached
 * with empty send/receive lists, and MPI_Wtime is a monotonic clock.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD      ((MPI_Comm)0)
#define MPI_SUCCESS         0
#define MPI_ANY_TAG         (-1)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE   ((MPI_Status *)0)

#define MPI_INT        ((MPI_Datatype)1)
#define MPI_DOUBLE     ((MPI_Datatype)2)
#define MPI_DOUBLE_INT ((MPI_Datatype)3)

#define MPI_SUM    ((MPI_Op)1)
#define MPI_MIN    ((MPI_Op)2)
#define MPI_MAX    ((MPI_Op)3)
#define MPI_MINLOC ((MPI_Op)4)
#define MPI_MAXLOC ((MPI_Op)5)

double MPI_Wtime(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count,
               MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *request);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *request);
int MPI_Waitall(int count, MPI_Request *requests, MPI_Status *statuses);
int MPI_Abort(MPI_Comm comm, int errorcode);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_MPI_SHIM_H */
