/*
 * oracle/solver2d.c -- CPU restatement of the reference's 2D Fortran solver
 * kernels (src/solver/src/*.F90), exported under the same bind(C) names and
 * argument lists, so that the reference's own C physics driver
 * (src/physics/src/*.c) links against it unchanged.
 *
 * TEST INFRASTRUCTURE. This file is the parity checker for the CUDA path;
 * no product code calls it.
 *
 * Restatement rules, so that results are bit-for-bit what the Fortran
 * computes without fused multiply-adds:
 *   - Fortran's column-major Q(nfields,n,n) indexing is kept:
 *     Q(f,i,j) (1-based) lives at [f-1 + nfields*((i-1) + n*(j-1))];
 *   - every expression keeps the Fortran source's operand order, with
 *     left-to-right evaluation of chains of * and +;
 *   - compiled with -O2 -ffp-contract=off -fno-fast-math.
 * Constants: gamma = 1.4 and gm1 = 0.4 are hard-coded in the kernels
 * exactly as the Fortran does (flux_2d_module.F90:41,82-83,
 * bc_2d_module.F90:213, solver_time_step_2d_module.F90:41-42); note that
 * the flux's pressure uses (gamma-1) = 0.3999999999999999 while its sound
 * speed uses the literal 0.4.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define QIDX(f, i, j, nf, n) ((f) + (nf) * (((i) - 1) + (n) * ((j) - 1)))

/* my_kinddefs.F90:412,424-426 */
static const double HALF = 0.5;
static const double PI_DP = 3.141592653589793238462643383279502884197;
static const double TWOPI_DP = 6.283185307179586476925286766559005768394;

/* ------------------------------------------------------------------ */
/* flux_2d_module.F90:32-60  flux_native_2d                           */
static void flux_native_2d(const double q[4], double flux[2][4])
{
    const double gamma = 1.4;
    double rho = q[0];
    double oneOrho = 1.0 / rho;
    double u = q[1] * oneOrho;
    double v = q[2] * oneOrho;
    double p = (gamma - 1.0) * (q[3] - 0.5 * rho * (u * u + v * v));

    flux[0][0] = q[1];
    flux[0][1] = q[1] * u + p;
    flux[0][2] = q[1] * v;
    flux[0][3] = u * (q[3] + p);

    flux[1][0] = q[2];
    flux[1][1] = q[2] * u;
    flux[1][2] = q[2] * v + p;
    flux[1][3] = v * (q[3] + p);
}

/* flux_2d_module.F90:13-29  flux_bc_2d */
static void flux_bc_2d(const double q[4], const double normal[2], double flux[4])
{
    double fl[2][4];
    flux_native_2d(q, fl);
    for (int k = 0; k < 4; ++k)
        flux[k] = fl[0][k] * normal[0] + fl[1][k] * normal[1];
}

/* flux_2d_module.F90:63-182  flux_roe_2d (HLL with Einfeldt bounds and a
 * Mach-weighted anti-dissipation term; non-unit normal, flux scaled by |n|) */
void oracle_flux_roe_2d(const double ql[4], const double qr[4],
                        const double norm[2], double flux[4])
{
    const double gamma = 1.4;
    const double gm1 = 0.4;
    double mag = sqrt(norm[0] * norm[0] + norm[1] * norm[1]);
    double nx = norm[0] / mag;
    double ny = norm[1] / mag;

    double rhol = ql[0];
    double oneOrhol = 1.0 / rhol;
    double ul = ql[1] * oneOrhol;
    double vl = ql[2] * oneOrhol;
    double El = ql[3] * oneOrhol;
    double pl = (gamma - 1.0) * (ql[3] - HALF * rhol * (ul * ul + vl * vl));
    double Hl = El + pl * oneOrhol;
    double unl = ul * nx + vl * ny;

    double rhor = qr[0];
    double oneOrhor = 1.0 / rhor;
    double ur = qr[1] * oneOrhor;
    double vr = qr[2] * oneOrhor;
    double Er = qr[3] * oneOrhor;
    double pr = (gamma - 1.0) * (qr[3] - HALF * rhor * (ur * ur + vr * vr));
    double Hr = Er + pr * oneOrhor;
    double unr = ur * nx + vr * ny;

    double srl = sqrt(rhol);
    double srr = sqrt(rhor);
    double roe_fact = srl + srr;
    double oneOroe_fact = 1.0 / roe_fact;
    double rhobar = sqrt(rhol * rhor);
    double ubar = (ul * srl + ur * srr) * oneOroe_fact;
    double vbar = (vl * srl + vr * srr) * oneOroe_fact;
    double Hbar = (Hl * srl + Hr * srr) * oneOroe_fact;
    double abar = sqrt(gm1 * (Hbar - HALF * (ubar * ubar + vbar * vbar)));
    double unbar = ubar * nx + vbar * ny;
    double Mnbar = unbar / abar;

    double eigp = unbar + abar;
    double eigm = unbar - abar;
    double eigp_max = unr + abar;
    double eigm_min = unl - abar;
    double b1, b2;
    if (eigp > 0.0 || eigp_max > 0.0)
        b1 = (eigp > eigp_max) ? eigp : eigp_max;
    else
        b1 = 0.0;
    if (eigm < 0.0 || eigm_min < 0.0)
        b2 = (eigm < eigm_min) ? eigm : eigm_min;
    else
        b2 = 0.0;

    double bcoeff = b1 * b2 / (b1 - b2);
    double delta1 = (rhor - rhol) - (pr - pl) / (abar * abar);
    double Mcoeff = 1.0 / (1.0 + fabs(Mnbar));
    double bM = bcoeff * Mcoeff;
    double fluxl, fluxr, disp;

    fluxl = ql[1] * nx + ql[2] * ny;
    fluxr = qr[1] * nx + qr[2] * ny;
    disp = bcoeff * (rhor - rhol) - bM * delta1;
    flux[0] = (b1 * fluxl - b2 * fluxr) / (b1 - b2) + disp;

    fluxl = (ql[1] * ul + pl) * nx + (ql[2] * ul) * ny;
    fluxr = (qr[1] * ur + pr) * nx + (qr[2] * ur) * ny;
    disp = bcoeff * (qr[1] - ql[1]) - bM * (delta1 * ubar + rhobar * (ur - ul - nx * (unr - unl)));
    flux[1] = (b1 * fluxl - b2 * fluxr) / (b1 - b2) + disp;

    fluxl = (ql[1] * vl) * nx + (ql[2] * vl + pl) * ny;
    fluxr = (qr[1] * vr) * nx + (qr[2] * vr + pr) * ny;
    disp = bcoeff * (qr[2] - ql[2]) - bM * (delta1 * vbar + rhobar * (vr - vl - ny * (unr - unl)));
    flux[2] = (b1 * fluxl - b2 * fluxr) / (b1 - b2) + disp;

    fluxl = (ql[3] + pl) * unl;
    fluxr = (qr[3] + pr) * unr;
    disp = bcoeff * (rhor * Hr - rhol * Hl) - bM * (delta1 * Hbar + rhobar * (Hr - Hl));
    flux[3] = (b1 * fluxl - b2 * fluxr) / (b1 - b2) + disp;

    for (int k = 0; k < 4; ++k)
        flux[k] = flux[k] * mag;
}

/* Extension with no reference counterpart: bc 3, a prescribed boundary
 * state (the supersonic inflow of the shock-bubble workload), set by
 * oracle_set_inflow. */
static double oracle_inflow[4];

void oracle_set_inflow(const double q[4])
{
    for (int k = 0; k < 4; k++) oracle_inflow[k] = q[k];
}

/* The post-shock state of a planar shock of Mach ms running into gas at
 * rest (rho1, p1), by the Rankine-Hugoniot relations: the inflow state of
 * the shock-bubble workload (an extension, restated from the relations). */
void oracle_shock_state(double gamma, double ms, double rho1, double p1, double out[4])
{
    double c1 = sqrt(gamma * p1 / rho1);
    double m2 = ms * ms;
    double rho2 = rho1 * (gamma + 1.0) * m2 / ((gamma - 1.0) * m2 + 2.0);
    double p2 = p1 * (1.0 + 2.0 * gamma / (gamma + 1.0) * (m2 - 1.0));
    double u2 = ms * c1 * (1.0 - rho1 / rho2);
    out[0] = rho2;
    out[1] = rho2 * u2;
    out[2] = 0.0;
    out[3] = p2 / (gamma - 1.0) + 0.5 * rho2 * u2 * u2;
}

/* bc_2d_module.F90:14-75  bc_2d (0: extrapolate, 1: slip wall, 2: no-slip;
 * 3: the prescribed state above, an extension) */
static void bc_2d(int bc_type, const double normal[2], const double Q[4], double Q_bc[4])
{
    const double gamma = 1.4;
    double gm1 = gamma - 1.0;
    double rho = Q[0];
    double oneOrho = 1.0 / rho;
    double u = Q[1] * oneOrho;
    double v = Q[2] * oneOrho;
    double p = gm1 * (Q[3] - 0.5 * rho * (u * u + v * v));
    (void)p;
    switch (bc_type) {
    case 0:
        for (int k = 0; k < 4; ++k) Q_bc[k] = Q[k];
        break;
    case 1: {
        double mag = sqrt(normal[0] * normal[0] + normal[1] * normal[1]);
        double nx = normal[0] / mag;
        double ny = normal[1] / mag;
        double U_dot_n = u * nx + v * ny;
        double ub = u - U_dot_n * nx;
        double vb = v - U_dot_n * ny;
        Q_bc[0] = Q[0];
        Q_bc[1] = Q[0] * ub;
        Q_bc[2] = Q[0] * vb;
        Q_bc[3] = Q[3];
        break;
    }
    case 2:
        Q_bc[0] = Q[0];
        Q_bc[1] = 0.0;
        Q_bc[2] = 0.0;
        Q_bc[3] = Q[3] - 0.5 * rho * (u * u + v * v);
        break;
    case 3:
        for (int k = 0; k < 4; k++) Q_bc[k] = oracle_inflow[k];
        break;
    default:
        /* The Fortran leaves Q_bc undefined for other types; the oracle
         * refuses them instead of inventing a value. */
        fprintf(stderr, "oracle bc_2d: unsupported bc type %d\n", bc_type);
        abort();
    }
}

/* bilinear_node_2d_module.F90:14-36 */
static void bilinear_node_2d(const double *g, const double nat[2], double out[2])
{
    double oneMxi = 0.5 * (1.0 - nat[0]);
    double onePxi = 0.5 * (1.0 + nat[0]);
    double oneMeta = 0.5 * (1.0 - nat[1]);
    double onePeta = 0.5 * (1.0 + nat[1]);
    for (int c = 0; c < 2; ++c)
        out[c] = g[c + 0] * oneMxi * oneMeta + g[c + 3] * onePxi * oneMeta +
                 g[c + 6] * oneMxi * onePeta + g[c + 9] * onePxi * onePeta;
}

/* Level-scaled subgrid spacing used by every edge-face kernel:
 * cell_h = h_base * (1/2**level) / n, e.g.
 * solver_residual_face_full_structured_2d_module.F90:239 */
static double cell_h_of(double h_base, int level, int n)
{
    return h_base * (1.0 / ldexp(1.0, level)) / (double)n;
}

static double sub_scale(int n) { return 2.0 / (double)n; }

/* ------------------------------------------------------------------ */
/* solver_residual_subgrid_2d_module.F90:32-164 */
static void residual_subgrid_2d(int nf, int n, const double *g, const double *Q, double *res)
{
    double s = sub_scale(n);
    double flux[4], nv[2], n1[2], n2[2], n3[2], n4[2];
    double a1[2], a2[2], a3[2], a4[2];

    for (int j = 1; j <= n; ++j) {
        a1[1] = s * (double)(j - 1) - 1.0;
        a2[1] = s * (double)j - 1.0;
        for (int i = 1; i <= n - 1; ++i) {
            a1[0] = s * (double)i - 1.0;
            a2[0] = s * (double)i - 1.0;
            bilinear_node_2d(g, a1, n1);
            bilinear_node_2d(g, a2, n2);
            nv[0] = n2[1] - n1[1];
            nv[1] = n1[0] - n2[0];
            oracle_flux_roe_2d(&Q[QIDX(0, i, j, nf, n)], &Q[QIDX(0, i + 1, j, nf, n)], nv, flux);
            for (int k = 0; k < 4; ++k) {
                res[QIDX(k, i, j, nf, n)] = res[QIDX(k, i, j, nf, n)] + flux[k];
                res[QIDX(k, i + 1, j, nf, n)] = res[QIDX(k, i + 1, j, nf, n)] - flux[k];
            }
        }
    }
    for (int j = 1; j <= n - 1; ++j) {
        a1[1] = s * (double)j - 1.0;
        a2[1] = s * (double)j - 1.0;
        for (int i = 1; i <= n; ++i) {
            a1[0] = s * (double)i - 1.0;
            a2[0] = s * (double)(i - 1) - 1.0;
            bilinear_node_2d(g, a1, n1);
            bilinear_node_2d(g, a2, n2);
            nv[0] = n2[1] - n1[1];
            nv[1] = n1[0] - n2[0];
            oracle_flux_roe_2d(&Q[QIDX(0, i, j, nf, n)], &Q[QIDX(0, i, j + 1, nf, n)], nv, flux);
            for (int k = 0; k < 4; ++k) {
                res[QIDX(k, i, j, nf, n)] = res[QIDX(k, i, j, nf, n)] + flux[k];
                res[QIDX(k, i, j + 1, nf, n)] = res[QIDX(k, i, j + 1, nf, n)] - flux[k];
            }
        }
    }
    for (int j = 1; j <= n; ++j) {
        double v1 = s * (double)(j - 1) - 1.0;
        double v2 = s * (double)j - 1.0;
        a1[1] = v1; a2[1] = v1; a3[1] = v2; a4[1] = v2;
        for (int i = 1; i <= n; ++i) {
            double w1 = s * (double)(i - 1) - 1.0;
            double w2 = s * (double)i - 1.0;
            a1[0] = w1; a2[0] = w2; a3[0] = w1; a4[0] = w2;
            bilinear_node_2d(g, a1, n1);
            bilinear_node_2d(g, a2, n2);
            bilinear_node_2d(g, a3, n3);
            bilinear_node_2d(g, a4, n4);
            double vec1[2] = {n4[0] - n1[0], n4[1] - n1[1]};
            double vec2[2] = {n3[0] - n2[0], n3[1] - n2[1]};
            double cr = vec1[0] * vec2[1] - vec1[1] * vec2[0];
            double volume = 0.5 * sqrt(cr * cr);
            for (int k = 0; k < 4; ++k)
                res[QIDX(k, i, j, nf, n)] = res[QIDX(k, i, j, nf, n)] / volume;
        }
    }
}

/* solver_residual_subgrid.F90:22-45 (dimension dispatch) */
void solver_residual_subgrid(int *dim, int *nfields, int *nelem_subgrid, int *type,
                             int *level, double *cell_geom, double *soln, double *res)
{
    (void)type; (void)level;
    if (*dim != 2) { fprintf(stderr, "oracle: 3D residual not restated\n"); abort(); }
    residual_subgrid_2d(*nfields, *nelem_subgrid, cell_geom, soln, res);
}

/* solver_residual_face_full_structured_2d_module.F90:199-273 */
static void residual_face_full_2d(int nf, int n, int side, int level, int ind_l_in, int ind_r_in,
                                  int dof, double h_base, const double *ql, const double *qr,
                                  double *res)
{
    int ind_l = ind_l_in + 1;
    int ind_r = ind_r_in + 1;
    double cell_h = cell_h_of(h_base, level, n);
    double nv[2], flux[4];
    double *rl = &res[ind_l_in];
    double *rr = &res[ind_r_in];
    if (side == 1) {
        nv[0] = cell_h; nv[1] = 0.0;
        for (int j = 1; j <= n; ++j) {
            oracle_flux_roe_2d(&ql[QIDX(0, n, j, nf, n)], &qr[QIDX(0, 1, j, nf, n)], nv, flux);
            if (ind_l < dof) for (int k = 0; k < 4; ++k) rl[QIDX(k, n, j, nf, n)] = rl[QIDX(k, n, j, nf, n)] + flux[k];
            if (ind_r < dof) for (int k = 0; k < 4; ++k) rr[QIDX(k, 1, j, nf, n)] = rr[QIDX(k, 1, j, nf, n)] - flux[k];
        }
    } else if (side == 3) {
        nv[0] = 0.0; nv[1] = cell_h;
        for (int i = 1; i <= n; ++i) {
            oracle_flux_roe_2d(&ql[QIDX(0, i, n, nf, n)], &qr[QIDX(0, i, 1, nf, n)], nv, flux);
            if (ind_l < dof) for (int k = 0; k < 4; ++k) rl[QIDX(k, i, n, nf, n)] = rl[QIDX(k, i, n, nf, n)] + flux[k];
            if (ind_r < dof) for (int k = 0; k < 4; ++k) rr[QIDX(k, i, 1, nf, n)] = rr[QIDX(k, i, 1, nf, n)] - flux[k];
        }
    }
}

/* solver_residual_face_full_structured.F90:32-68 (dimension dispatch) */
void solver_residual_face_full_structured(int *dim, int *nfields, int *nelem_subgrid, int *side,
                                          int *level, int *type_l, int *type_r, int *ind_l,
                                          int *ind_r, int *dof, double *h_base, double *xlo,
                                          double *ylo, double *zlo, double *ql, double *qr,
                                          double *res)
{
    (void)type_l; (void)type_r; (void)xlo; (void)ylo; (void)zlo;
    if (*dim != 2) { fprintf(stderr, "oracle: 3D face not restated\n"); abort(); }
    residual_face_full_2d(*nfields, *nelem_subgrid, *side, *level, *ind_l, *ind_r, *dof,
                          *h_base, ql, qr, res);
}

/* solver_residual_face_full_hang_structured_2d.F90:34-128
 * coarse quad on the left, two fine quads on the right; index-based pairing:
 * coarse edge cell j meets edge cell j of each fine quad, fine-level cell_h. */
void solver_residual_face_full_hang_structured_2d(
    int *nfields, int *nelem_subgrid, int *side, int *level_l, int *level_r,
    int *type_l, int *type_r1, int *type_r2, int *ind_l_in, int *ind_r1_in, int *ind_r2_in,
    int *dof, double *h_base, double *xlo, double *ylo, double *zlo,
    double *ql, double *qr_1, double *qr_2, double *res)
{
    (void)level_l; (void)type_l; (void)type_r1; (void)type_r2; (void)xlo; (void)ylo; (void)zlo;
    int nf = *nfields, n = *nelem_subgrid;
    int ind_l = *ind_l_in + 1, ind_r1 = *ind_r1_in + 1, ind_r2 = *ind_r2_in + 1;
    double cell_h = cell_h_of(*h_base, *level_r, n);
    double *rl = &res[*ind_l_in], *rr1 = &res[*ind_r1_in], *rr2 = &res[*ind_r2_in];
    double nv[2], flux[4];
    if (*side == 1) {
        nv[0] = cell_h; nv[1] = 0.0;
        for (int j = 1; j <= n; ++j) {
            oracle_flux_roe_2d(&ql[QIDX(0, n, j, nf, n)], &qr_1[QIDX(0, 1, j, nf, n)], nv, flux);
            if (ind_l < *dof) for (int k = 0; k < 4; ++k) rl[QIDX(k, n, j, nf, n)] = rl[QIDX(k, n, j, nf, n)] + flux[k];
            if (ind_r1 < *dof) for (int k = 0; k < 4; ++k) rr1[QIDX(k, 1, j, nf, n)] = rr1[QIDX(k, 1, j, nf, n)] - flux[k];
            oracle_flux_roe_2d(&ql[QIDX(0, n, j, nf, n)], &qr_2[QIDX(0, 1, j, nf, n)], nv, flux);
            if (ind_l < *dof) for (int k = 0; k < 4; ++k) rl[QIDX(k, n, j, nf, n)] = rl[QIDX(k, n, j, nf, n)] + flux[k];
            if (ind_r2 < *dof) for (int k = 0; k < 4; ++k) rr2[QIDX(k, 1, j, nf, n)] = rr2[QIDX(k, 1, j, nf, n)] - flux[k];
        }
    } else if (*side == 3) {
        nv[0] = 0.0; nv[1] = cell_h;
        for (int i = 1; i <= n; ++i) {
            oracle_flux_roe_2d(&ql[QIDX(0, i, n, nf, n)], &qr_1[QIDX(0, i, 1, nf, n)], nv, flux);
            if (ind_l < *dof) for (int k = 0; k < 4; ++k) rl[QIDX(k, i, n, nf, n)] = rl[QIDX(k, i, n, nf, n)] + flux[k];
            if (ind_r1 < *dof) for (int k = 0; k < 4; ++k) rr1[QIDX(k, i, 1, nf, n)] = rr1[QIDX(k, i, 1, nf, n)] - flux[k];
            oracle_flux_roe_2d(&ql[QIDX(0, i, n, nf, n)], &qr_2[QIDX(0, i, 1, nf, n)], nv, flux);
            if (ind_l < *dof) for (int k = 0; k < 4; ++k) rl[QIDX(k, i, n, nf, n)] = rl[QIDX(k, i, n, nf, n)] + flux[k];
            if (ind_r2 < *dof) for (int k = 0; k < 4; ++k) rr2[QIDX(k, i, 1, nf, n)] = rr2[QIDX(k, i, 1, nf, n)] - flux[k];
        }
    }
}

/* solver_residual_face_hang_full_structured_2d.F90:34-128
 * two fine quads on the left, coarse quad on the right (mirror of the above). */
void solver_residual_face_hang_full_structured_2d(
    int *nfields, int *nelem_subgrid, int *side, int *level_l, int *level_r,
    int *type_l1, int *type_l2, int *type_r, int *ind_l1_in, int *ind_l2_in, int *ind_r_in,
    int *dof, double *h_base, double *xlo, double *ylo, double *zlo,
    double *ql_1, double *ql_2, double *qr, double *res)
{
    (void)level_r; (void)type_l1; (void)type_l2; (void)type_r; (void)xlo; (void)ylo; (void)zlo;
    int nf = *nfields, n = *nelem_subgrid;
    int ind_l1 = *ind_l1_in + 1, ind_l2 = *ind_l2_in + 1, ind_r = *ind_r_in + 1;
    double cell_h = cell_h_of(*h_base, *level_l, n);
    double *rl1 = &res[*ind_l1_in], *rl2 = &res[*ind_l2_in], *rr = &res[*ind_r_in];
    double nv[2], flux[4];
    if (*side == 1) {
        nv[0] = cell_h; nv[1] = 0.0;
        for (int j = 1; j <= n; ++j) {
            oracle_flux_roe_2d(&ql_1[QIDX(0, n, j, nf, n)], &qr[QIDX(0, 1, j, nf, n)], nv, flux);
            if (ind_l1 < *dof) for (int k = 0; k < 4; ++k) rl1[QIDX(k, n, j, nf, n)] = rl1[QIDX(k, n, j, nf, n)] + flux[k];
            if (ind_r < *dof) for (int k = 0; k < 4; ++k) rr[QIDX(k, 1, j, nf, n)] = rr[QIDX(k, 1, j, nf, n)] - flux[k];
            oracle_flux_roe_2d(&ql_2[QIDX(0, n, j, nf, n)], &qr[QIDX(0, 1, j, nf, n)], nv, flux);
            if (ind_l2 < *dof) for (int k = 0; k < 4; ++k) rl2[QIDX(k, n, j, nf, n)] = rl2[QIDX(k, n, j, nf, n)] + flux[k];
            if (ind_r < *dof) for (int k = 0; k < 4; ++k) rr[QIDX(k, 1, j, nf, n)] = rr[QIDX(k, 1, j, nf, n)] - flux[k];
        }
    } else if (*side == 3) {
        nv[0] = 0.0; nv[1] = cell_h;
        for (int i = 1; i <= n; ++i) {
            oracle_flux_roe_2d(&ql_1[QIDX(0, i, n, nf, n)], &qr[QIDX(0, i, 1, nf, n)], nv, flux);
            if (ind_l1 < *dof) for (int k = 0; k < 4; ++k) rl1[QIDX(k, i, n, nf, n)] = rl1[QIDX(k, i, n, nf, n)] + flux[k];
            if (ind_r < *dof) for (int k = 0; k < 4; ++k) rr[QIDX(k, i, 1, nf, n)] = rr[QIDX(k, i, 1, nf, n)] - flux[k];
            oracle_flux_roe_2d(&ql_2[QIDX(0, i, n, nf, n)], &qr[QIDX(0, i, 1, nf, n)], nv, flux);
            if (ind_l2 < *dof) for (int k = 0; k < 4; ++k) rl2[QIDX(k, i, n, nf, n)] = rl2[QIDX(k, i, n, nf, n)] + flux[k];
            if (ind_r < *dof) for (int k = 0; k < 4; ++k) rr[QIDX(k, i, 1, nf, n)] = rr[QIDX(k, i, 1, nf, n)] - flux[k];
        }
    }
}

/* subgrid_index_2d_module.F90:14-46 */
static void subgrid_index_2d(int ind, int end_ind, int side, int *i, int *j)
{
    switch (side) {
    case 0: *i = 1; *j = ind; break;
    case 1: *i = end_ind; *j = ind; break;
    case 2: *i = ind; *j = 1; break;
    case 3: *i = ind; *j = end_ind; break;
    default: *i = 1; *j = 1; break;
    }
}

/* solver_residual_bc_structured_2d_module.F90:31-88 */
static void residual_bc_2d(int nf, int n, int side, int level, int bc, double h_base,
                           const double *soln, double *res)
{
    double cell_h = cell_h_of(h_base, level, n);
    double nv[2] = {0.0, 0.0}, Q_bc[4], flux[4];
    switch (side) {
    case 0: nv[0] = -cell_h; break;
    case 1: nv[0] = cell_h; break;
    case 2: nv[1] = -cell_h; break;
    case 3: nv[1] = cell_h; break;
    }
    for (int m = 1; m <= n; ++m) {
        int i, j;
        subgrid_index_2d(m, n, side, &i, &j);
        bc_2d(bc, nv, &soln[QIDX(0, i, j, nf, n)], Q_bc);
        flux_bc_2d(Q_bc, nv, flux);
        for (int k = 0; k < 4; ++k)
            res[QIDX(k, i, j, nf, n)] = res[QIDX(k, i, j, nf, n)] + flux[k];
    }
}

/* solver_residual_bc_structured.F90:28-56 (dimension dispatch) */
void solver_residual_bc_structured(int *dim, int *nfields, int *nelem_subgrid, int *side,
                                   int *type, int *level, int *bc, double *h_base, double *xlo,
                                   double *ylo, double *zlo, double *soln, double *res)
{
    (void)type; (void)xlo; (void)ylo; (void)zlo;
    if (*dim != 2) { fprintf(stderr, "oracle: 3D bc not restated\n"); abort(); }
    residual_bc_2d(*nfields, *nelem_subgrid, *side, *level, *bc, *h_base, soln, res);
}

/* solver_time_step_2d_module.F90:26-122 */
static void time_step_2d(int nf, int n, const double *g, const double *Q, double cfl, double *dt)
{
    const double gamma = 1.4;
    const double gm1 = 0.4;
    double s = sub_scale(n);
    double a1[2], a2[2], a3[2], a4[2], n1[2], n2[2], n3[2], n4[2];
    for (int j = 1; j <= n; ++j) {
        double v1 = s * (double)(j - 1) - 1.0;
        double v2 = s * (double)j - 1.0;
        a1[1] = v1; a2[1] = v1; a3[1] = v2; a4[1] = v2;
        for (int i = 1; i <= n; ++i) {
            double w1 = s * (double)(i - 1) - 1.0;
            double w2 = s * (double)i - 1.0;
            a1[0] = w1; a2[0] = w2; a3[0] = w1; a4[0] = w2;
            bilinear_node_2d(g, a1, n1);
            bilinear_node_2d(g, a2, n2);
            bilinear_node_2d(g, a3, n3);
            bilinear_node_2d(g, a4, n4);
            double vec1[2] = {n4[0] - n1[0], n4[1] - n1[1]};
            double vec2[2] = {n3[0] - n2[0], n3[1] - n2[1]};
            double cr = vec1[0] * vec2[1] - vec1[1] * vec2[0];
            double volume = 0.5 * sqrt(cr * cr);
            const double *q = &Q[QIDX(0, i, j, nf, n)];
            double oneOrho = 1.0 / q[0];
            double u = q[1] * oneOrho;
            double v = q[2] * oneOrho;
            double V2 = u * u + v * v;
            double pOverRho = gm1 * (q[3] * oneOrho - HALF * V2);
            double c = sqrt(gamma * pOverRho);
            double eig = sqrt(V2) + c;
            double cand = cfl * sqrt(volume) / eig;
            if (cand < *dt) *dt = cand;
        }
    }
}

/* solver_time_step.F90:22-46 (dimension dispatch) */
void solver_time_step(int *dim, int *nfields, int *nelem_subgrid, int *type, int *level,
                      double *cell_geom, double *soln, double *cfl, double *dt)
{
    (void)type; (void)level;
    if (*dim != 2) { fprintf(stderr, "oracle: 3D dt not restated\n"); abort(); }
    time_step_2d(*nfields, *nelem_subgrid, cell_geom, soln, *cfl, dt);
}

/* solver_tag_feature.F90:9-52 + tagging_methods_module.F90:14-71 */
void solver_tag_feature(int *ntag, int *tag_methods, double *tag_tolerances, int *dim,
                        int *unstructured, int *nfields, int *nsub_elem, int *cell_type,
                        double *elem_h, double *elem_xyz, double *elem_soln, int *tag)
{
    (void)unstructured; (void)cell_type; (void)elem_h; (void)elem_xyz;
    int ncells = 1;
    for (int d = 0; d < *dim; ++d) ncells *= *nsub_elem;
    *tag = 0;
    for (int m = 0; m < *ntag; ++m) {
        double tol = tag_tolerances[m];
        if (tag_methods[m] == 1) {
            for (int c = 0; c < ncells; ++c)
                if (elem_soln[*nfields * c] <= tol) { *tag = 1; break; }
        } else if (tag_methods[m] == 2) {
            for (int c = 0; c < ncells; ++c)
                if (elem_soln[*nfields * c] >= tol) { *tag = 1; break; }
        }
    }
}

/* initial_condition_2d_module.F90:12-131 (IC 0 free stream, IC 1 Shu vortex
 * at the origin, beta 3, a 0.5) + initial_boundary_2d_module.F90:15-36 */
void solver_initialize_quadrant(int *initial_condition, int *dim, int *unstructured, int *nfields,
                                int *nelem_subgrid, int *cell_type, double *h, double *cell_geom,
                                double *Q, double *mach, double *alpha, double *beta,
                                double *gamma, double *density, double *pressure)
{
    (void)h;
    if (*dim != 2) { fprintf(stderr, "oracle: 3D IC not restated\n"); abort(); }
    int nf = *nfields, n = *nelem_subgrid;
    *cell_type = 0;
    if (*unstructured == 1 && fabs(cell_geom[0]) < 10.0) *cell_type = 1;

    double gm1 = *gamma - 1.0;
    double oneOgm1 = 1.0 / gm1;
    double RT0 = *pressure / *density;
    double C_0 = sqrt(*gamma * RT0);
    double V_0 = *mach * C_0;
    double u_in = V_0 * cos(*alpha * PI_DP / 180.0) * cos(*beta * PI_DP / 180.0);
    double v_in = V_0 * sin(*alpha * PI_DP / 180.0) * cos(*beta * PI_DP / 180.0);
    double rhou = *density * u_in;
    double rhov = *density * v_in;
    double rhoe = (*pressure * oneOgm1) + HALF * *density * (u_in * u_in + v_in * v_in);
    double time = 0.0;

    if (*initial_condition == 0) {
        for (int j = 1; j <= n; ++j)
            for (int i = 1; i <= n; ++i) {
                Q[QIDX(0, i, j, nf, n)] = *density;
                Q[QIDX(1, i, j, nf, n)] = rhou;
                Q[QIDX(2, i, j, nf, n)] = rhov;
                Q[QIDX(3, i, j, nf, n)] = rhoe;
            }
    } else if (*initial_condition == 1) {
        double xo = 0.0, yo = 0.0;
        xo = xo + u_in * time;
        yo = yo + v_in * time;
        double a = 0.5, beta_L = 3.0;
        double two_a = 2.0 * a;
        double dT1 = -(gm1 * beta_L * beta_L) / (16.0 * a * *gamma * PI_DP * PI_DP);
        double s = sub_scale(n);
        double nat[2], node[2];
        for (int j = 1; j <= n; ++j) {
            double v1 = s * (double)(j - 1) - 1.0;
            double v2 = s * (double)j - 1.0;
            nat[1] = 0.5 * (v1 + v2);
            for (int i = 1; i <= n; ++i) {
                double w1 = s * (double)(i - 1) - 1.0;
                double w2 = s * (double)i - 1.0;
                nat[0] = 0.5 * (w1 + w2);
                bilinear_node_2d(cell_geom, nat, node);
                double u = u_in, v = v_in;
                double radius2 = (node[0] - xo) * (node[0] - xo) + (node[1] - yo) * (node[1] - yo);
                double dT = dT1 * exp(two_a * (1.0 - radius2));
                double rho = pow(1.0 + dT, oneOgm1);
                double ff = beta_L / TWOPI_DP * exp(a * (1.0 - radius2));
                u = u - (node[1] - yo) * ff;
                v = v + (node[0] - xo) * ff;
                double p = *pressure + pow(rho, *gamma) - 1.0;
                Q[QIDX(0, i, j, nf, n)] = rho;
                Q[QIDX(1, i, j, nf, n)] = rho * u;
                Q[QIDX(2, i, j, nf, n)] = rho * v;
                Q[QIDX(3, i, j, nf, n)] = p * oneOgm1 + HALF * rho * (u * u + v * v);
            }
        }
    }
}

/* solver_refine_operator_2d.F90:28-55: every child receives the parent patch */
void solver_refine_operator_2d(int *unstructured, int *numfields, int *nsub_elem, int *cell_type,
                               double *h, double *geom, double *soln, double *uc1, double *uc2,
                               double *uc3, double *uc4)
{
    (void)unstructured; (void)cell_type; (void)h; (void)geom;
    int m = *numfields * *nsub_elem * *nsub_elem;
    for (int k = 0; k < m; ++k) { uc1[k] = soln[k]; uc2[k] = soln[k]; uc3[k] = soln[k]; uc4[k] = soln[k]; }
}

/* solver_coarsen_operator_2d.F90:29-53: same-index average of the children */
void solver_coarsen_operator_2d(int *unstructured, int *numfields, int *nsub_elem, int *cell_type,
                                double *h, double *geom, double *uc1, double *uc2, double *uc3,
                                double *uc4, double *soln)
{
    (void)unstructured; (void)cell_type; (void)h; (void)geom;
    int m = *numfields * *nsub_elem * *nsub_elem;
    for (int k = 0; k < m; ++k) {
        double s = uc1[k] + uc2[k] + uc3[k] + uc4[k];
        soln[k] = 0.25 * s;
    }
}
