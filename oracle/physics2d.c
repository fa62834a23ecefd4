/*
 * oracle/physics2d.c -- CPU restatement of the reference's C physics driver
 * for one rank (src/physics/src/*.c), on top of the Fortran restatement in
 * solver2d.c.
 *
 * TEST INFRASTRUCTURE. It is the parity checker for the CUDA path and the
 * CPU baseline port; no product code calls it. The reference's own driver
 * sources, compiled unmodified from the reference tree by oracle/Makefile
 * into oracle/_ref/, pin this restatement bit for bit (tests/test_oracle.py).
 *
 * Functions and what they restate:
 *   oracle_rhs        physics_rhs_structured.c:19-283
 *   oracle_time_step  physics_time_step.c:16-49
 *   oracle_norm       physics_norm_residual.c:15-56
 *   oracle_evolve     physics_go.c:16-132 + physics_runge_kutta_interface.c:23-357
 *                     + rk_time_integrators.c:22-540 on one rank (MPI
 *                     reductions are the identity), plus the final-time
 *                     extension used by the benchmark workloads (dt clipped
 *                     to reach final_time exactly; no reference counterpart).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void solver_residual_subgrid(int *dim, int *nfields, int *nelem_subgrid, int *type, int *level,
                             double *cell_geom, double *soln, double *res);
void solver_residual_bc_structured(int *dim, int *nfields, int *nelem_subgrid, int *side, int *type,
                                   int *level, int *bc, double *h_base, double *xlo, double *ylo,
                                   double *zlo, double *soln, double *res);
void solver_residual_face_full_structured(int *dim, int *nfields, int *nelem_subgrid, int *side,
                                          int *level, int *type_l, int *type_r, int *ind_l, int *ind_r,
                                          int *dof, double *h_base, double *xlo, double *ylo,
                                          double *zlo, double *ql, double *qr, double *res);
void solver_residual_face_full_hang_structured_2d(
    int *nfields, int *nelem_subgrid, int *side, int *level_l, int *level_r, int *type_l,
    int *type_r1, int *type_r2, int *ind_l_in, int *ind_r1_in, int *ind_r2_in, int *dof,
    double *h_base, double *xlo, double *ylo, double *zlo, double *ql, double *qr_1, double *qr_2,
    double *res);
void solver_residual_face_hang_full_structured_2d(
    int *nfields, int *nelem_subgrid, int *side, int *level_l, int *level_r, int *type_l1,
    int *type_l2, int *type_r, int *ind_l1_in, int *ind_l2_in, int *ind_r_in, int *dof,
    double *h_base, double *xlo, double *ylo, double *zlo, double *ql_1, double *ql_2, double *qr,
    double *res);
void solver_time_step(int *dim, int *nfields, int *nelem_subgrid, int *type, int *level,
                      double *cell_geom, double *soln, double *cfl, double *dt);

typedef struct {
    int nelem_subgrid;
    int time_scheme;
    int time_steps;
    int regrid_interval, checkpoint_interval, visualization_interval; /* <= 0: never */
    int bc[4];
    double dt;       /* cap */
    double cfl;      /* effective (scaled) CFL */
    double h_base;   /* coarse_grid_h */
    double final_time;
    double time;     /* in/out: simulated time (extension) */
} oracle_config_t;

/* physics_rhs_structured.c:19-283 (2D, 3 ints per cell, 11 per face) */
void oracle_rhs(const oracle_config_t *cfg, int ncell, const int *cell_info, int nface,
                const int *face_info, double *geom, int dof, double *soln, double *rhs)
{
    int dim = 2, nfields = 4, n = cfg->nelem_subgrid, dofv = dof;
    int ncorners = 12;
    double h_base = cfg->h_base;
    double xlo[2] = {0, 0}, ylo[2] = {0, 0}, zlo[2] = {0, 0};
    for (int i = 0; i < dof; i++) rhs[i] = 0.0;
    for (int f = 0; f < nface; f++) {
        const int *fi = &face_info[11 * f];
        int facetype = fi[0], side = fi[1], cell = fi[2];
        int type = cell_info[3 * cell + 0], level = cell_info[3 * cell + 1], ind = cell_info[3 * cell + 2];
        int ql[4], qr[4], type_l[4], type_r[4], ind_l[4], ind_r[4];
        if (side % 2 == 0) {
            for (int k = 0; k < 4; k++) {
                ql[k] = fi[3 + k];
                type_l[k] = ql[k] >= 0 ? cell_info[3 * ql[k] + 0] : -1;
                ind_l[k] = ql[k] >= 0 ? cell_info[3 * ql[k] + 2] : -1;
            }
            qr[0] = cell;
            type_r[0] = cell_info[3 * cell + 0];
            ind_r[0] = cell_info[3 * cell + 2];
        } else {
            for (int k = 0; k < 4; k++) {
                qr[k] = fi[3 + k];
                type_r[k] = qr[k] >= 0 ? cell_info[3 * qr[k] + 0] : -1;
                ind_r[k] = qr[k] >= 0 ? cell_info[3 * qr[k] + 2] : -1;
            }
            ql[0] = cell;
            type_l[0] = cell_info[3 * cell + 0];
            ind_l[0] = cell_info[3 * cell + 2];
        }
        int level_l = cell_info[3 * ql[0] + 1];
        int level_r = cell_info[3 * qr[0] + 1];
        int side_plus;
        switch (facetype) {
        case 1: {
            int bcv = cfg->bc[side];
            solver_residual_bc_structured(&dim, &nfields, &n, &side, &type, &level, &bcv, &h_base,
                                          &xlo[0], &ylo[0], &zlo[0], &soln[ind], &rhs[ind]);
            break;
        }
        case 2:
            side_plus = (side % 2 == 0) ? side + 1 : side;
            solver_residual_face_full_structured(&dim, &nfields, &n, &side_plus, &level_l, &type_l[0],
                                                 &type_r[0], &ind_l[0], &ind_r[0], &dofv, &h_base, xlo,
                                                 ylo, zlo, &soln[ind_l[0]], &soln[ind_r[0]], rhs);
            break;
        case 3:
            if (side % 2 == 0) {
                side_plus = side + 1;
                solver_residual_face_hang_full_structured_2d(
                    &nfields, &n, &side_plus, &level_l, &level_r, &type_l[0], &type_l[1], &type_r[0],
                    &ind_l[0], &ind_l[1], &ind_r[0], &dofv, &h_base, xlo, ylo, zlo, &soln[ind_l[0]],
                    &soln[ind_l[1]], &soln[ind_r[0]], rhs);
            } else {
                side_plus = side;
                solver_residual_face_full_hang_structured_2d(
                    &nfields, &n, &side_plus, &level_l, &level_r, &type_l[0], &type_r[0], &type_r[1],
                    &ind_l[0], &ind_r[0], &ind_r[1], &dofv, &h_base, xlo, ylo, zlo, &soln[ind_l[0]],
                    &soln[ind_r[0]], &soln[ind_r[1]], rhs);
            }
            break;
        default:
            fprintf(stderr, "oracle_rhs: unsupported face type %d\n", facetype);
            abort();
        }
    }
    for (int c = 0; c < ncell; c++) {
        int type = cell_info[3 * c + 0], level = cell_info[3 * c + 1], off = cell_info[3 * c + 2];
        solver_residual_subgrid(&dim, &nfields, &n, &type, &level, &geom[ncorners * c], &soln[off],
                                &rhs[off]);
    }
    for (int i = 0; i < dof; i++) rhs[i] *= -1.0;
}

/* physics_time_step.c:16-49 */
void oracle_time_step(const oracle_config_t *cfg, int ncell, const int *cell_info, double *geom,
                      double *soln, double *dt)
{
    int dim = 2, nfields = 4, n = cfg->nelem_subgrid;
    double cfl = cfg->cfl;
    for (int c = 0; c < ncell; c++) {
        int type = cell_info[3 * c + 0], level = cell_info[3 * c + 1], off = cell_info[3 * c + 2];
        solver_time_step(&dim, &nfields, &n, &type, &level, &geom[12 * c], &soln[off], &cfl, dt);
    }
}

/* physics_norm_residual.c:15-56 (2D) */
double oracle_norm(int n, int ncell, const int *cell_info, const double *res)
{
    double s = 0.0;
    int nftm = 4 * n * n;
    for (int c = 0; c < ncell; c++) {
        const double *r = &res[cell_info[3 * c + 2]];
        for (int j = 0; j < nftm; j++) s += r[j] * r[j];
    }
    return s;
}

static int hit(int istep, int interval) { return interval > 0 && istep % interval == 0; }

/* physics_go.c:66-69 + physics_runge_kutta_interface.c:23-357 on one rank.
 * Returns the number of steps taken; *resnorm gets sqrt(sum k^2) of the
 * last stage (rk_*: MPI_Allreduce(SUM) then sqrt). */
int oracle_evolve(oracle_config_t *cfg, int ncell, const int *cell_info, int nface,
                  const int *face_info, double *geom, int dof, double *Q, int *istep, int *regrid,
                  int *visualize, int *checkpoint, int *evolve_solution, double *resnorm,
                  double *dt_last)
{
    int n = cfg->nelem_subgrid;
    int ts = cfg->time_scheme;
    if (*istep >= cfg->time_steps) {
        *evolve_solution = 0;
        return 0;
    }
    size_t bytes = sizeof(double) * (size_t)(dof > 0 ? dof : 1);
    double *k1 = malloc(bytes), *k2 = malloc(bytes), *k3 = malloc(bytes), *k4 = malloc(bytes);
    double *Qs = malloc(bytes);
    int steps = 0, go = 1;
    *resnorm = -1.0;
    while (go) {
        double dt = cfg->dt;
        if (ts != 2) oracle_time_step(cfg, ncell, cell_info, geom, Q, &dt);
        if (cfg->final_time > 0.0) {
            double rem = cfg->final_time - cfg->time;
            if (rem < dt) dt = rem;
            if (dt < 0.0) dt = 0.0;
        }
        double rn = 0.0;
        switch (ts) {
        case 1: {
            double beta1 = 1.0 * dt;
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k1);
            rn = oracle_norm(n, ncell, cell_info, k1);
            for (int i = 0; i < dof; ++i) Q[i] = Q[i] + beta1 * k1[i];
            break;
        }
        case 2: {
            double alpha1 = 1.0 * dt, beta1 = 0.5 * dt, beta2 = 0.5 * dt;
            for (int i = 0; i < dof; ++i) Qs[i] = Q[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k1);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + alpha1 * k1[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k2);
            rn = oracle_norm(n, ncell, cell_info, k2);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + beta1 * k1[i] + beta2 * k2[i];
            break;
        }
        case 3: {
            double alpha1 = 1.00 * dt, alpha21 = 0.25 * dt, alpha22 = 0.25 * dt;
            double beta1 = 1.0 / 6.0 * dt, beta2 = 1.0 / 6.0 * dt, beta3 = 2.0 / 3.0 * dt;
            for (int i = 0; i < dof; ++i) Qs[i] = Q[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k1);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + alpha1 * k1[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k2);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + alpha21 * k1[i] + alpha22 * k2[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k3);
            rn = oracle_norm(n, ncell, cell_info, k3);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + beta1 * k1[i] + beta2 * k2[i] + beta3 * k3[i];
            break;
        }
        case 4: {
            double alpha1 = 0.5 * dt, alpha2 = 0.5 * dt, alpha3 = 1.0 * dt, beta1 = 1.0 / 6.0 * dt;
            for (int i = 0; i < dof; ++i) Qs[i] = Q[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k1);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + alpha1 * k1[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k2);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + alpha2 * k2[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k3);
            for (int i = 0; i < dof; ++i) Q[i] = Qs[i] + alpha3 * k3[i];
            oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k4);
            rn = oracle_norm(n, ncell, cell_info, k4);
            for (int i = 0; i < dof; ++i)
                Q[i] = Qs[i] + beta1 * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
            break;
        }
        case 5: {
            const double ra[5] = {0.0, -567301805773.0 / 1357537059087.0,
                                  -2404267990393.0 / 2016746695238.0,
                                  -3550918686646.0 / 2091501179385.0,
                                  -1275806237668.0 / 842570457699.0};
            const double rb[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                                  1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                                  2277821191437.0 / 14882151754819.0};
            for (int st = 0; st < 5; ++st) {
                oracle_rhs(cfg, ncell, cell_info, nface, face_info, geom, dof, Q, k1);
                rn = oracle_norm(n, ncell, cell_info, k1);
                for (int i = 0; i < dof; ++i) {
                    Qs[i] = (st == 0) ? dt * k1[i] : Qs[i] * ra[st] + dt * k1[i];
                    Q[i] = Q[i] + rb[st] * Qs[i];
                }
            }
            break;
        }
        default:
            fprintf(stderr, "oracle_evolve: unsupported time scheme %d\n", ts);
            abort();
        }
        *resnorm = sqrt(rn);
        *dt_last = dt;
        cfg->time = cfg->time + dt;
        *istep += 1;
        steps += 1;
        if (*istep >= cfg->time_steps) go = 0;
        if (hit(*istep, cfg->regrid_interval)) { go = 0; *regrid = 1; }
        if (hit(*istep, cfg->checkpoint_interval)) { go = 0; *checkpoint = 1; }
        if (hit(*istep, cfg->visualization_interval)) { go = 0; *visualize = 1; }
        if (cfg->final_time > 0.0 && cfg->time >= cfg->final_time) { go = 0; *evolve_solution = 0; }
    }
    free(k1); free(k2); free(k3); free(k4); free(Qs);
    return steps;
}
