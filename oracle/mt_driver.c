/*
 * mt_driver.c -- runs the reference's own physics_go
 * (src/physics/src/physics_go.c:16-132) on P ranks as P threads of one
 * process, over the thread MPI stand-in (mpi_shim/mpi_threads.c): the
 * reference's multi-rank path with its ghost exchange, the CPU baseline's
 * "MPI CPU path". oracle_mt_evolve enters through physics_evolve_interface
 * (physics_evolve_interface.c:15-53) instead, which in a -D_GPU_ build of
 * the reference hands every rank to physics_go_gpu.
 * TEST INFRASTRUCTURE: nothing in the product links it.
 *
 * Each rank gets the arrays the reference's AMR driver would hand it
 * (external_t, amr_external.c:211-508): its local quads then its ghost quads,
 * the faces that touch its quads, the (cell, rank) send and receive lists
 * and the per-cell record sizes.
 */
#include <pthread.h>
#include <stdlib.h>

#include "mpi.h"

void physics_go(int *dim, int *unstructured, int *nfields, int *nelem_subgrid, int *ncell, int *nghost,
                int *nface, int *dof, int *cell_info, int *face_info, int *nsend, int *nrecv, int *send, int *recv,
                int *sizes, double *geom, double *soln, int *istep, int *regrid, int *visualize, int *checkpoint,
                int *evolve_solution, MPI_Comm mpicomm_ext, double *total_time, double *compute_time,
                double *residual_time);
void physics_evolve_interface(int *dim, int *unstructured, int *nfields, int *nelem_subgrid, int *ncell,
                              int *nghost, int *nface, int *dof, int *cell_info, int *face_info, int *nsend,
                              int *nrecv, int *send, int *recv, int *sizes, double *geom, double *soln, int *istep,
                              int *regrid, int *visualize, int *checkpoint, int *evolve_solution,
                              MPI_Comm mpicomm_ext, double *total_time, double *compute_time,
                              double *residual_time);
int oracle_mt_init(int size);
void oracle_mt_finalize(void);
void oracle_mt_set_rank(int r);

typedef struct {
    int ncell, nghost, nface, dof, nsend, nrecv;
    int *cell_info, *face_info, *send, *recv, *sizes;
    double *geom, *soln;
    int istep, regrid, visualize, checkpoint, evolve_solution;
    double total_time, compute_time, residual_time;
    double wall;  /* seconds this rank spent in physics_go */
} oracle_mt_rank_t;

typedef struct {
    int rank, n, via_interface;
    oracle_mt_rank_t *r;
} mt_task;

static void *mt_rank_main(void *arg)
{
    mt_task *t = (mt_task *)arg;
    oracle_mt_rank_t *r = t->r;
    int dim = 2, uns = 0, nf = 4, n = t->n;
    oracle_mt_set_rank(t->rank);
    double t0 = MPI_Wtime();
    if (t->via_interface)
        physics_evolve_interface(&dim, &uns, &nf, &n, &r->ncell, &r->nghost, &r->nface, &r->dof, r->cell_info,
                                 r->face_info, &r->nsend, &r->nrecv, r->send, r->recv, r->sizes, r->geom, r->soln,
                                 &r->istep, &r->regrid, &r->visualize, &r->checkpoint, &r->evolve_solution,
                                 (MPI_Comm)0, &r->total_time, &r->compute_time, &r->residual_time);
    else
        physics_go(&dim, &uns, &nf, &n, &r->ncell, &r->nghost, &r->nface, &r->dof, r->cell_info, r->face_info,
                   &r->nsend, &r->nrecv, r->send, r->recv, r->sizes, r->geom, r->soln, &r->istep, &r->regrid,
                   &r->visualize, &r->checkpoint, &r->evolve_solution, (MPI_Comm)0, &r->total_time,
                   &r->compute_time, &r->residual_time);
    r->wall = MPI_Wtime() - t0;
    return NULL;
}

static int mt_run(int nranks, int n, oracle_mt_rank_t *ranks, int via_interface)
{
    if (oracle_mt_init(nranks)) return 1;
    pthread_t *th = (pthread_t *)calloc((size_t)nranks, sizeof(pthread_t));
    mt_task *tk = (mt_task *)calloc((size_t)nranks, sizeof(mt_task));
    int rc = (th && tk) ? 0 : 1;
    int started = 0;
    for (int r = 0; r < nranks && !rc; r++) {
        tk[r].rank = r;
        tk[r].n = n;
        tk[r].via_interface = via_interface;
        tk[r].r = &ranks[r];
        if (pthread_create(&th[r], NULL, mt_rank_main, &tk[r]) != 0) rc = 1;
        else started++;
    }
    for (int r = 0; r < started; r++) pthread_join(th[r], NULL);
    free(th);
    free(tk);
    oracle_mt_finalize();
    return rc || started != nranks;
}

/* physics_go on every rank, one thread each; returns 0 when all ran. */
int oracle_mt_go(int nranks, int n, oracle_mt_rank_t *ranks) { return mt_run(nranks, n, ranks, 0); }

/* physics_evolve_interface on every rank, one thread each. */
int oracle_mt_evolve(int nranks, int n, oracle_mt_rank_t *ranks) { return mt_run(nranks, n, ranks, 1); }
