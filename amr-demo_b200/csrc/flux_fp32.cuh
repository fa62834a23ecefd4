// flux_fp32.cuh -- the same face physics as flux_fp64.cuh (the reference's
// flux_roe_2d, flux_2d_module.F90:63-182, and bc_2d + flux_bc_2d,
// bc_2d_module.F90:14-75) in FP32 with fast reciprocals and square roots,
// for the FP32-flux form. The algebra is rearranged where it saves work
// (one reciprocal of b1-b2, sqrt(rhol*rhor) = sqrt(rhol)*sqrt(rhor)); the
// form's error against the FP64 result is measured, not assumed.
#pragma once

namespace amrgpu {

__device__ __forceinline__ void roe_flux_fp32(const float ql[4], const float qr[4], float n0,
                                              float n1, float flux[4])
{
    const float gm1p = 0.4f;  // (gamma - 1) for the pressure
    const float gm1 = 0.4f;
    float mag = sqrtf(n0 * n0 + n1 * n1);
    float inv_mag = __frcp_rn(mag);
    float nx = n0 * inv_mag;
    float ny = n1 * inv_mag;

    float rhol = ql[0];
    float oneOrhol = __frcp_rn(rhol);
    float ul = ql[1] * oneOrhol;
    float vl = ql[2] * oneOrhol;
    float pl = gm1p * (ql[3] - 0.5f * rhol * (ul * ul + vl * vl));
    float Hl = (ql[3] + pl) * oneOrhol;
    float unl = ul * nx + vl * ny;

    float rhor = qr[0];
    float oneOrhor = __frcp_rn(rhor);
    float ur = qr[1] * oneOrhor;
    float vr = qr[2] * oneOrhor;
    float pr = gm1p * (qr[3] - 0.5f * rhor * (ur * ur + vr * vr));
    float Hr = (qr[3] + pr) * oneOrhor;
    float unr = ur * nx + vr * ny;

    float srl = sqrtf(rhol);
    float srr = sqrtf(rhor);
    float oneOroe = __frcp_rn(srl + srr);
    float rhobar = srl * srr;
    float ubar = (ul * srl + ur * srr) * oneOroe;
    float vbar = (vl * srl + vr * srr) * oneOroe;
    float Hbar = (Hl * srl + Hr * srr) * oneOroe;
    float a2 = gm1 * (Hbar - 0.5f * (ubar * ubar + vbar * vbar));
    float abar = sqrtf(a2);
    float unbar = ubar * nx + vbar * ny;
    float Mnbar = unbar * __frcp_rn(abar);

    float eigp = unbar + abar;
    float eigm = unbar - abar;
    float b1 = fmaxf(fmaxf(eigp, unr + abar), 0.0f);
    float b2 = fminf(fminf(eigm, unl - abar), 0.0f);
    float inv_db = __frcp_rn(b1 - b2);
    float bcoeff = b1 * b2 * inv_db;
    float delta1 = (rhor - rhol) - (pr - pl) * __frcp_rn(a2);
    float bM = bcoeff * __frcp_rn(1.0f + fabsf(Mnbar));
    float dun = unr - unl;

    float fluxl, fluxr, disp;
    fluxl = ql[1] * nx + ql[2] * ny;
    fluxr = qr[1] * nx + qr[2] * ny;
    disp = bcoeff * (rhor - rhol) - bM * delta1;
    flux[0] = ((b1 * fluxl - b2 * fluxr) * inv_db + disp) * mag;

    fluxl = (ql[1] * ul + pl) * nx + (ql[2] * ul) * ny;
    fluxr = (qr[1] * ur + pr) * nx + (qr[2] * ur) * ny;
    disp = bcoeff * (qr[1] - ql[1]) - bM * (delta1 * ubar + rhobar * (ur - ul - nx * dun));
    flux[1] = ((b1 * fluxl - b2 * fluxr) * inv_db + disp) * mag;

    fluxl = (ql[1] * vl) * nx + (ql[2] * vl + pl) * ny;
    fluxr = (qr[1] * vr) * nx + (qr[2] * vr + pr) * ny;
    disp = bcoeff * (qr[2] - ql[2]) - bM * (delta1 * vbar + rhobar * (vr - vl - ny * dun));
    flux[2] = ((b1 * fluxl - b2 * fluxr) * inv_db + disp) * mag;

    fluxl = (ql[3] + pl) * unl;
    fluxr = (qr[3] + pr) * unr;
    disp = bcoeff * (rhor * Hr - rhol * Hl) - bM * (delta1 * Hbar + rhobar * (Hr - Hl));
    flux[3] = ((b1 * fluxl - b2 * fluxr) * inv_db + disp) * mag;
}

__device__ __forceinline__ void bc_flux_fp32(int bc, const float q[4], float n0, float n1,
                                             const float qin[4], float flux[4])
{
    float qb[4];
    float oneOrho = __frcp_rn(q[0]);
    float u = q[1] * oneOrho;
    float v = q[2] * oneOrho;
    if (bc == 1) {
        float inv_mag = rsqrtf(n0 * n0 + n1 * n1);
        float nx = n0 * inv_mag, ny = n1 * inv_mag;
        float Un = u * nx + v * ny;
        qb[0] = q[0];
        qb[1] = q[0] * (u - Un * nx);
        qb[2] = q[0] * (v - Un * ny);
        qb[3] = q[3];
    } else if (bc == 2) {
        qb[0] = q[0];
        qb[1] = 0.0f;
        qb[2] = 0.0f;
        qb[3] = q[3] - 0.5f * q[0] * (u * u + v * v);
    } else if (bc == 3) {
        qb[0] = qin[0]; qb[1] = qin[1]; qb[2] = qin[2]; qb[3] = qin[3];
    } else {
        qb[0] = q[0]; qb[1] = q[1]; qb[2] = q[2]; qb[3] = q[3];
    }
    float oor = __frcp_rn(qb[0]);
    float ub = qb[1] * oor, vb = qb[2] * oor;
    float p = 0.4f * (qb[3] - 0.5f * qb[0] * (ub * ub + vb * vb));
    flux[0] = qb[1] * n0 + qb[2] * n1;
    flux[1] = (qb[1] * ub + p) * n0 + (qb[2] * ub) * n1;
    flux[2] = (qb[1] * vb) * n0 + (qb[2] * vb + p) * n1;
    flux[3] = (ub * n0 + vb * n1) * (qb[3] + p);
}

}  // namespace amrgpu
