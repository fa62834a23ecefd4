/*
 * physics_go_gpu.h -- the header the reference's physics layer includes
 * when built with -D_GPU_ (src/physics/src/physics_evolve_interface.h:16-17)
 * and that the reference never shipped. It declares physics_go_gpu with
 * physics_go's signature (src/physics/src/physics_go.h:59); libamrgpu.so
 * (include/amrgpu.h) provides the definition.
 *
 * The communicator is accepted as the caller's MPI_Comm; libamrgpu runs one
 * rank per process and does not use it (multi-rank ghost exchange is not
 * part of this library: nsend/nrecv/nghost must be 0).
 */
#ifndef PHYSICS_GO_GPU_H
#define PHYSICS_GO_GPU_H

#include <mpi.h>

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

#ifdef __cplusplus
}
#endif

#endif /* PHYSICS_GO_GPU_H */
