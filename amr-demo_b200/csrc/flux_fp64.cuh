// flux_fp64.cuh -- the reference's face physics in FP64, operation for
// operation. Included only by translation units built with -fmad=false, so
// that no multiply-add is contracted and every result is the IEEE-rounded
// value the reference's Fortran produces without FMA:
//   roe_flux_fp64   flux_2d_module.F90:63-182 (flux_roe_2d)
//   bc_flux_fp64    bc_2d_module.F90:14-75 + flux_2d_module.F90:13-60
//   cfl_candidate   solver_time_step_2d_module.F90:106-116
// gamma = 1.4 and gm1 = 0.4 are hard-coded exactly as there; the flux's
// pressure uses (gamma - 1) = 0.3999999999999999, its sound speed 0.4.
#pragma once

namespace amrgpu {

__device__ __forceinline__ void roe_flux_fp64(const double ql[4], const double qr[4],
                                              double n0, double n1, double flux[4])
{
    const double gamma = 1.4;
    const double gm1 = 0.4;
    const double half = 0.5;
    double mag = sqrt(n0 * n0 + n1 * n1);
    double nx = n0 / mag;
    double ny = n1 / mag;

    double rhol = ql[0];
    double oneOrhol = 1.0 / rhol;
    double ul = ql[1] * oneOrhol;
    double vl = ql[2] * oneOrhol;
    double El = ql[3] * oneOrhol;
    double pl = (gamma - 1.0) * (ql[3] - half * rhol * (ul * ul + vl * vl));
    double Hl = El + pl * oneOrhol;
    double unl = ul * nx + vl * ny;

    double rhor = qr[0];
    double oneOrhor = 1.0 / rhor;
    double ur = qr[1] * oneOrhor;
    double vr = qr[2] * oneOrhor;
    double Er = qr[3] * oneOrhor;
    double pr = (gamma - 1.0) * (qr[3] - half * rhor * (ur * ur + vr * vr));
    double Hr = Er + pr * oneOrhor;
    double unr = ur * nx + vr * ny;

    double srl = sqrt(rhol);
    double srr = sqrt(rhor);
    double oneOroe_fact = 1.0 / (srl + srr);
    double rhobar = sqrt(rhol * rhor);
    double ubar = (ul * srl + ur * srr) * oneOroe_fact;
    double vbar = (vl * srl + vr * srr) * oneOroe_fact;
    double Hbar = (Hl * srl + Hr * srr) * oneOroe_fact;
    double abar = sqrt(gm1 * (Hbar - half * (ubar * ubar + vbar * vbar)));
    double unbar = ubar * nx + vbar * ny;
    double Mnbar = unbar / abar;

    double eigp = unbar + abar;
    double eigm = unbar - abar;
    double eigp_max = unr + abar;
    double eigm_min = unl - abar;
    double b1 = (eigp > 0.0 || eigp_max > 0.0) ? ((eigp > eigp_max) ? eigp : eigp_max) : 0.0;
    double b2 = (eigm < 0.0 || eigm_min < 0.0) ? ((eigm < eigm_min) ? eigm : eigm_min) : 0.0;

    double bcoeff = b1 * b2 / (b1 - b2);
    double delta1 = (rhor - rhol) - (pr - pl) / (abar * abar);
    double Mcoeff = 1.0 / (1.0 + fabs(Mnbar));
    double bM = bcoeff * Mcoeff;
    double db = b1 - b2;
    double fluxl, fluxr, disp;

    fluxl = ql[1] * nx + ql[2] * ny;
    fluxr = qr[1] * nx + qr[2] * ny;
    disp = bcoeff * (rhor - rhol) - bM * delta1;
    flux[0] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;

    fluxl = (ql[1] * ul + pl) * nx + (ql[2] * ul) * ny;
    fluxr = (qr[1] * ur + pr) * nx + (qr[2] * ur) * ny;
    disp = bcoeff * (qr[1] - ql[1]) - bM * (delta1 * ubar + rhobar * (ur - ul - nx * (unr - unl)));
    flux[1] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;

    fluxl = (ql[1] * vl) * nx + (ql[2] * vl + pl) * ny;
    fluxr = (qr[1] * vr) * nx + (qr[2] * vr + pr) * ny;
    disp = bcoeff * (qr[2] - ql[2]) - bM * (delta1 * vbar + rhobar * (vr - vl - ny * (unr - unl)));
    flux[2] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;

    fluxl = (ql[3] + pl) * unl;
    fluxr = (qr[3] + pr) * unr;
    disp = bcoeff * (rhor * Hr - rhol * Hl) - bM * (delta1 * Hbar + rhobar * (Hr - Hl));
    flux[3] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;
}

// Per-cell primitive record shared by the four faces of a cell:
// [0] rho [1] rho*u [2] rho*v [3] rho*E [4] u [5] v [6] p [7] H [8] sqrt(rho),
// each computed by exactly the expression flux_roe_2d uses
// (flux_2d_module.F90:93-99, 113-118), so reusing them is bit-exact.
__device__ __forceinline__ void cell_prims_fp64(const double q[4], double P[9])
{
    const double gamma = 1.4;
    const double half = 0.5;
    double rho = q[0];
    double oneOrho = 1.0 / rho;
    double u = q[1] * oneOrho;
    double v = q[2] * oneOrho;
    double E = q[3] * oneOrho;
    double p = (gamma - 1.0) * (q[3] - half * rho * (u * u + v * v));
    P[0] = q[0];
    P[1] = q[1];
    P[2] = q[2];
    P[3] = q[3];
    P[4] = u;
    P[5] = v;
    P[6] = p;
    P[7] = E + p * oneOrho;
    P[8] = sqrt(rho);
}

// flux_roe_2d on primitive records. For an axis-aligned normal (one
// component exactly zero) |n| = sqrt(n0*n0) is |n0| exactly in IEEE
// round-to-nearest and n0/|n0| = +-1, n1/|n0| = n1 (a signed zero), so the
// shortcut returns the same bits as the general path.
__device__ __forceinline__ void roe_flux_prim_fp64(const double *L, const double *R, double n0, double n1,
                                                   double flux[4])
{
    const double gm1 = 0.4;
    const double half = 0.5;
    double mag, nx, ny;
    if (n1 == 0.0 && fabs(n0) > 1e-150) {
        mag = fabs(n0);
        nx = n0 > 0.0 ? 1.0 : -1.0;
        ny = n1;
    } else if (n0 == 0.0 && fabs(n1) > 1e-150) {
        mag = fabs(n1);
        nx = n0;
        ny = n1 > 0.0 ? 1.0 : -1.0;
    } else {
        mag = sqrt(n0 * n0 + n1 * n1);
        nx = n0 / mag;
        ny = n1 / mag;
    }
    const double rhol = L[0], ul = L[4], vl = L[5], pl = L[6], Hl = L[7], srl = L[8];
    const double rhor = R[0], ur = R[4], vr = R[5], pr = R[6], Hr = R[7], srr = R[8];
    double unl = ul * nx + vl * ny;
    double unr = ur * nx + vr * ny;
    double oneOroe_fact = 1.0 / (srl + srr);
    double rhobar = sqrt(rhol * rhor);
    double ubar = (ul * srl + ur * srr) * oneOroe_fact;
    double vbar = (vl * srl + vr * srr) * oneOroe_fact;
    double Hbar = (Hl * srl + Hr * srr) * oneOroe_fact;
    double abar = sqrt(gm1 * (Hbar - half * (ubar * ubar + vbar * vbar)));
    double unbar = ubar * nx + vbar * ny;
    double Mnbar = unbar / abar;
    double eigp = unbar + abar;
    double eigm = unbar - abar;
    double eigp_max = unr + abar;
    double eigm_min = unl - abar;
    double b1 = (eigp > 0.0 || eigp_max > 0.0) ? ((eigp > eigp_max) ? eigp : eigp_max) : 0.0;
    double b2 = (eigm < 0.0 || eigm_min < 0.0) ? ((eigm < eigm_min) ? eigm : eigm_min) : 0.0;
    double bcoeff = b1 * b2 / (b1 - b2);
    double delta1 = (rhor - rhol) - (pr - pl) / (abar * abar);
    double Mcoeff = 1.0 / (1.0 + fabs(Mnbar));
    double bM = bcoeff * Mcoeff;
    double db = b1 - b2;
    double fluxl, fluxr, disp;

    fluxl = L[1] * nx + L[2] * ny;
    fluxr = R[1] * nx + R[2] * ny;
    disp = bcoeff * (rhor - rhol) - bM * delta1;
    flux[0] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;

    fluxl = (L[1] * ul + pl) * nx + (L[2] * ul) * ny;
    fluxr = (R[1] * ur + pr) * nx + (R[2] * ur) * ny;
    disp = bcoeff * (R[1] - L[1]) - bM * (delta1 * ubar + rhobar * (ur - ul - nx * (unr - unl)));
    flux[1] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;

    fluxl = (L[1] * vl) * nx + (L[2] * vl + pl) * ny;
    fluxr = (R[1] * vr) * nx + (R[2] * vr + pr) * ny;
    disp = bcoeff * (R[2] - L[2]) - bM * (delta1 * vbar + rhobar * (vr - vl - ny * (unr - unl)));
    flux[2] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;

    fluxl = (L[3] + pl) * unl;
    fluxr = (R[3] + pr) * unr;
    disp = bcoeff * (rhor * Hr - rhol * Hl) - bM * (delta1 * Hbar + rhobar * (Hr - Hl));
    flux[3] = ((b1 * fluxl - b2 * fluxr) / db + disp) * mag;
}

// Boundary face: ghost state of bc_2d, then the physical flux F.n of
// flux_bc_2d. bc 3 (extension, no reference counterpart): prescribed state
// qin, used for supersonic inflow.
__device__ __forceinline__ void bc_flux_fp64(int bc, const double q[4], double n0, double n1,
                                             const double qin[4], double flux[4])
{
    const double gamma = 1.4;
    double qb[4];
    double rho = q[0];
    double oneOrho = 1.0 / rho;
    double u = q[1] * oneOrho;
    double v = q[2] * oneOrho;
    if (bc == 1) {
        double mag = sqrt(n0 * n0 + n1 * n1);
        double nx = n0 / mag;
        double ny = n1 / mag;
        double U_dot_n = u * nx + v * ny;
        double ub = u - U_dot_n * nx;
        double vb = v - U_dot_n * ny;
        qb[0] = q[0];
        qb[1] = q[0] * ub;
        qb[2] = q[0] * vb;
        qb[3] = q[3];
    } else if (bc == 2) {
        qb[0] = q[0];
        qb[1] = 0.0;
        qb[2] = 0.0;
        qb[3] = q[3] - 0.5 * rho * (u * u + v * v);
    } else if (bc == 3) {
        qb[0] = qin[0]; qb[1] = qin[1]; qb[2] = qin[2]; qb[3] = qin[3];
    } else {
        qb[0] = q[0]; qb[1] = q[1]; qb[2] = q[2]; qb[3] = q[3];
    }
    // flux_native_2d
    double r = qb[0];
    double oor = 1.0 / r;
    double ub2 = qb[1] * oor;
    double vb2 = qb[2] * oor;
    double p = (gamma - 1.0) * (qb[3] - 0.5 * r * (ub2 * ub2 + vb2 * vb2));
    double fx0 = qb[1], fx1 = qb[1] * ub2 + p, fx2 = qb[1] * vb2, fx3 = ub2 * (qb[3] + p);
    double fy0 = qb[2], fy1 = qb[2] * ub2, fy2 = qb[2] * vb2 + p, fy3 = vb2 * (qb[3] + p);
    flux[0] = fx0 * n0 + fy0 * n1;
    flux[1] = fx1 * n0 + fy1 * n1;
    flux[2] = fx2 * n0 + fy2 * n1;
    flux[3] = fx3 * n0 + fy3 * n1;
}

// One cell's CFL step candidate: cfl*sqrt(volume)/(|V| + c).
__device__ __forceinline__ double cfl_candidate_fp64(const double q[4], double volume, double cfl)
{
    const double gamma = 1.4;
    const double gm1 = 0.4;
    double oneOrho = 1.0 / q[0];
    double u = q[1] * oneOrho;
    double v = q[2] * oneOrho;
    double V2 = u * u + v * v;
    double pOverRho = gm1 * (q[3] * oneOrho - 0.5 * V2);
    double c = sqrt(gamma * pOverRho);
    double eig = sqrt(V2) + c;
    return cfl * sqrt(volume) / eig;
}

}  // namespace amrgpu
