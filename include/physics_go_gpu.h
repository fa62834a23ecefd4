/*
 * physics_go_gpu.h -- the header the reference's physics layer includes
 * when built with -D_GPU_ (src/physics/src/physics_evolve_interface.h:16-17)
 * and that the reference never shipped. It declares physics_go_gpu with
 * physics_go's signature (src/physics/src/physics_go.h:59); libamrgpu.so
 * (include/amrgpu.h) provides the definition.
 *
 * libamrgpu links no MPI. For multi-rank calls (ghost quads) it needs three
 * operations on the caller's communicator: the ghost-record exchange of
 * physics_mpi_real_to_ghost (physics_mpi.c:47-122) and the MIN / SUM
 * all-reduces of the time step and the residual norm. This header compiles
 * them against the caller's own <mpi.h> and installs them with
 * amrgpu_set_comm_ops when the library that includes it is loaded, so the
 * reference's -D_GPU_ build needs no source change. Define
 * AMRGPU_NO_MPI_ADAPTER to leave them out (and install your own).
 *
 * Include this header before amrgpu.h in a translation unit that includes
 * both: it sets the ABI's communicator type to MPI_Comm.
 */
#ifndef PHYSICS_GO_GPU_H
#define PHYSICS_GO_GPU_H

#include <mpi.h>
#include <stdlib.h>

#ifndef AMRGPU_COMM_T
#define AMRGPU_COMM_T MPI_Comm
#endif
#include "amrgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

void physics_go_gpu(int *dim, int *unstructured, int *nfields, int *nelem_subgrid,
                    int *ncell, int *nghost, int *nface, int *dof, int *cell_info,
                    int *face_info, int *nsend, int *nrecv, int *send, int *recv,
                    int *sizes, double *geom, double *soln, int *istep, int *regrid,
                    int *visualize, int *checkpoint, int *evolve_solution,
                    MPI_Comm mpicomm_ext, double *total_time, double *compute_time,
                    double *residual_time);

#ifndef AMRGPU_NO_MPI_ADAPTER

static int amrgpu_mpi_rank_(MPI_Comm comm, int *rank)
{
    return MPI_Comm_rank(comm, rank) == MPI_SUCCESS ? 0 : 1;
}

/* One message per run of consecutive list entries with the same peer, the
 * grouping physics_mpi_real_to_ghost uses (receives posted first, then the
 * sends, then one wait for all). Receives match any tag, sends use 35, as
 * there. */
static int amrgpu_mpi_exchange_(MPI_Comm comm, int nsend, const int *send, int nrecv, const int *recv,
                                int stride, int record_doubles, const double *sendbuf, double *recvbuf)
{
    MPI_Request *req = (MPI_Request *)malloc(sizeof(MPI_Request) * (size_t)(nsend + nrecv + 1));
    int nreq = 0, k = 0, ok = 1;
    if (!req) return 1;
    while (k < nrecv && ok) {
        const int peer = recv[stride * k + 1];
        int e = k + 1;
        while (e < nrecv && recv[stride * e + 1] == peer) ++e;
        ok = MPI_Irecv(recvbuf + (size_t)k * (size_t)record_doubles, (e - k) * record_doubles, MPI_DOUBLE, peer,
                       MPI_ANY_TAG, comm, &req[nreq++]) == MPI_SUCCESS;
        k = e;
    }
    k = 0;
    while (k < nsend && ok) {
        const int peer = send[stride * k + 1];
        int e = k + 1;
        while (e < nsend && send[stride * e + 1] == peer) ++e;
        ok = MPI_Isend((void *)(sendbuf + (size_t)k * (size_t)record_doubles), (e - k) * record_doubles,
                       MPI_DOUBLE, peer, 35, comm, &req[nreq++]) == MPI_SUCCESS;
        k = e;
    }
    if (nreq > 0 && MPI_Waitall(nreq, req, MPI_STATUSES_IGNORE) != MPI_SUCCESS) ok = 0;
    free(req);
    return ok ? 0 : 1;
}

static int amrgpu_mpi_allreduce_(MPI_Comm comm, double *value, int op)
{
    double in = *value;
    MPI_Op o = (op == 0) ? MPI_MIN : (op == 1) ? MPI_SUM : MPI_MAX;
    return MPI_Allreduce(&in, value, 1, MPI_DOUBLE, o, comm) == MPI_SUCCESS ? 0 : 1;
}

__attribute__((constructor)) static void amrgpu_mpi_adapter_install_(void)
{
    amrgpu_comm_ops_t ops;
    ops.rank = amrgpu_mpi_rank_;
    ops.exchange = amrgpu_mpi_exchange_;
    ops.allreduce = amrgpu_mpi_allreduce_;
    amrgpu_set_comm_ops(&ops);
}

#endif /* AMRGPU_NO_MPI_ADAPTER */

#ifdef __cplusplus
}
#endif

#endif /* PHYSICS_GO_GPU_H */
