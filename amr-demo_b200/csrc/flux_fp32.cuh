// flux_fp32.cuh -- the same face physics as flux_fp64.cuh (the reference's
// flux_roe_2d, flux_2d_module.F90:63-182, and bc_2d + flux_bc_2d,
// bc_2d_module.F90:14-75) in FP32 with fast reciprocals and square roots,
// for the FP32-flux form. The algebra is rearranged where it saves work
// (one reciprocal of b1-b2, sqrt(rhol*rhor) = sqrt(rhol)*sqrt(rhor)); the
// form's error against the FP64 result is measured, not assumed.
#pragma once

namespace amrgpu {

// Reciprocal by the SFU's approximation (rcp.approx.ftz.f32, one MUFU
// operation, within an ulp or so) instead of the correctly rounded sequence.
__device__ __forceinline__ float frcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 1/sqrt(x) by the SFU's approximation (rsqrt.approx.ftz.f32).
__device__ __forceinline__ float frsqrt(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void roe_flux_fp32(const float ql[4], const float qr[4], float n0,
                                              float n1, float flux[4])
{
    const float gm1p = 0.4f;  // (gamma - 1) for the pressure
    const float gm1 = 0.4f;
    float mag = sqrtf(n0 * n0 + n1 * n1);
    float inv_mag = frcp(mag);
    float nx = n0 * inv_mag;
    float ny = n1 * inv_mag;

    float rhol = ql[0];
    float oneOrhol = frcp(rhol);
    float ul = ql[1] * oneOrhol;
    float vl = ql[2] * oneOrhol;
    float pl = gm1p * (ql[3] - 0.5f * rhol * (ul * ul + vl * vl));
    float Hl = (ql[3] + pl) * oneOrhol;
    float unl = ul * nx + vl * ny;

    float rhor = qr[0];
    float oneOrhor = frcp(rhor);
    float ur = qr[1] * oneOrhor;
    float vr = qr[2] * oneOrhor;
    float pr = gm1p * (qr[3] - 0.5f * rhor * (ur * ur + vr * vr));
    float Hr = (qr[3] + pr) * oneOrhor;
    float unr = ur * nx + vr * ny;

    float srl = sqrtf(rhol);
    float srr = sqrtf(rhor);
    float oneOroe = frcp(srl + srr);
    float rhobar = srl * srr;
    float ubar = (ul * srl + ur * srr) * oneOroe;
    float vbar = (vl * srl + vr * srr) * oneOroe;
    float Hbar = (Hl * srl + Hr * srr) * oneOroe;
    float a2 = gm1 * (Hbar - 0.5f * (ubar * ubar + vbar * vbar));
    float abar = sqrtf(a2);
    float unbar = ubar * nx + vbar * ny;
    float Mnbar = unbar * frcp(abar);

    float eigp = unbar + abar;
    float eigm = unbar - abar;
    float b1 = fmaxf(fmaxf(eigp, unr + abar), 0.0f);
    float b2 = fminf(fminf(eigm, unl - abar), 0.0f);
    float inv_db = frcp(b1 - b2);
    float bcoeff = b1 * b2 * inv_db;
    float delta1 = (rhor - rhol) - (pr - pl) * frcp(a2);
    float bM = bcoeff * frcp(1.0f + fabsf(Mnbar));
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

// Every operation of the per-cell record and of the axis-aligned flux below
// is written with an explicitly rounded intrinsic (__fmul_rn, __fadd_rn,
// __fsub_rn, __fmaf_rn) or an SFU instruction in inline PTX, so that the
// compiler cannot contract or reorder them differently at different
// inlined call sites: a face that two quads evaluate from their own sides
// (or one kernel in two places) gets bit-identical values, which exact
// conservation needs.
__device__ __forceinline__ float fsqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Per-cell FP32 record (8 floats, two float4 loads):
// [0] rho [1] u [2] v [3] p [4] H [5] sqrt(rho) [6] rho*u [7] rho*v.
// rho*E + p is recovered as rho*H.
__device__ __forceinline__ void cell_prims_fp32(const double q[4], float P[8])
{
    const float rho = __double2float_rn(q[0]);
    const float ru = __double2float_rn(q[1]), rv = __double2float_rn(q[2]), rE = __double2float_rn(q[3]);
    const float oneOrho = frcp(rho);
    const float u = __fmul_rn(ru, oneOrho), v = __fmul_rn(rv, oneOrho);
    const float ke = __fmul_rn(__fmul_rn(0.5f, rho), __fmaf_rn(u, u, __fmul_rn(v, v)));
    const float p = __fmul_rn(0.4f, __fsub_rn(rE, ke));
    P[0] = rho;
    P[1] = u;
    P[2] = v;
    P[3] = p;
    P[4] = __fmul_rn(__fadd_rn(rE, p), oneOrho);
    P[5] = fsqrt_approx(rho);
    P[6] = ru;
    P[7] = rv;
}

// Lane arithmetic for the axis-aligned flux below: one face per lane
// (float) or two faces per lane in packed pairs (float2, sm_100's paired
// FP32 add / multiply / fused multiply-add, one instruction for both
// halves). Every operation is an explicitly rounded intrinsic, so the
// compiler cannot contract or reorder it, and a float2 half gets exactly
// the bits the float version gives for the same inputs. Min, max, absolute
// value and the SFU approximations act per half.
struct LaneF1 {
    using T = float;
    static __device__ __forceinline__ T c(float v) { return v; }
    static __device__ __forceinline__ T add(T a, T b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ T sub(T a, T b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ T mul(T a, T b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ T fma(T a, T b, T d) { return __fmaf_rn(a, b, d); }
    static __device__ __forceinline__ T max(T a, T b) { return fmaxf(a, b); }
    static __device__ __forceinline__ T min(T a, T b) { return fminf(a, b); }
    static __device__ __forceinline__ T abs(T a) { return fabsf(a); }
    static __device__ __forceinline__ T rcp(T a) { return frcp(a); }
    static __device__ __forceinline__ T rsqrt(T a) { return frsqrt(a); }
};

struct LaneF2 {
    using T = float2;
    static __device__ __forceinline__ T c(float v) { return make_float2(v, v); }
    static __device__ __forceinline__ T add(T a, T b) { return __fadd2_rn(a, b); }
    // a - b = RN(a + (-1) b): the same single rounding as a subtraction
    static __device__ __forceinline__ T sub(T a, T b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
    static __device__ __forceinline__ T mul(T a, T b) { return __fmul2_rn(a, b); }
    static __device__ __forceinline__ T fma(T a, T b, T d) { return __ffma2_rn(a, b, d); }
    static __device__ __forceinline__ T max(T a, T b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
    static __device__ __forceinline__ T min(T a, T b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
    static __device__ __forceinline__ T abs(T a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
    static __device__ __forceinline__ T rcp(T a) { return make_float2(frcp(a.x), frcp(a.y)); }
    static __device__ __forceinline__ T rsqrt(T a) { return make_float2(frsqrt(a.x), frsqrt(a.y)); }
};

// One side of an axis-aligned face in the face's frame: normal and
// tangential velocity (n, t) and momentum (mn, mt); (u, v) for a face with
// normal +x, (v, u) for normal +y.
template <typename T>
struct AxisSide {
    T rho, n, t, p, H, sr, mn, mt;
};

// flux_roe_2d (flux_2d_module.F90:63-182) for a face with positive normal
// of length h, L on the low side, in the face's frame. The algebra is
// arranged for fused operations: with hinv = h/(b1-b2) the flux rows are
// h*(b1 fl - b2 fr)/(b1-b2) + h*bcoeff*jump - h*bM*corr
//   = hb1 fl - hb2 fr + hbc jump - hbM corr,
// hb1 = b1 hinv, hb2 = b2 hinv, hbc = b1 hb2 = h bcoeff and
// hbM = hbc abar/(abar + |un|) = h bM (Mcoeff = 1/(1+|un/a|)); the wave
// speeds b1 = max(max(un, unr) + a, 0) and b2 = min(min(un, unl) - a, 0)
// equal the reference's max/min of the sums (rounding is monotone); 1/a^2
// is the square of the SFU's 1/sqrt(a^2). Out: mass, normal-momentum,
// tangential-momentum and energy rows.
template <typename Op>
__device__ __forceinline__ void roe_flux_rot(const AxisSide<typename Op::T> &L, const AxisSide<typename Op::T> &R,
                                             typename Op::T h, typename Op::T out[4])
{
    using T = typename Op::T;
    const T inv = Op::rcp(Op::add(L.sr, R.sr));
    const T rhobar = Op::mul(L.sr, R.sr);
    const T nbar = Op::mul(Op::fma(L.n, L.sr, Op::mul(R.n, R.sr)), inv);
    const T tbar = Op::mul(Op::fma(L.t, L.sr, Op::mul(R.t, R.sr)), inv);
    const T Hbar = Op::mul(Op::fma(L.H, L.sr, Op::mul(R.H, R.sr)), inv);
    const T q2 = Op::fma(nbar, nbar, Op::mul(tbar, tbar));
    const T a2 = Op::fma(Op::c(-0.2f), q2, Op::mul(Op::c(0.4f), Hbar));
    const T ra = Op::rsqrt(a2);
    const T abar = Op::mul(a2, ra);
    const T b1 = Op::max(Op::add(Op::max(nbar, R.n), abar), Op::c(0.0f));
    const T b2 = Op::min(Op::sub(Op::min(nbar, L.n), abar), Op::c(0.0f));
    const T hinv = Op::mul(h, Op::rcp(Op::sub(b1, b2)));
    const T hb1 = Op::mul(b1, hinv), hb2 = Op::mul(b2, hinv);
    const T hbc = Op::mul(b1, hb2);
    const T drho = Op::sub(R.rho, L.rho);
    const T delta1 = Op::fma(Op::sub(L.p, R.p), Op::mul(ra, ra), drho);
    const T hbM = Op::mul(Op::mul(hbc, abar), Op::rcp(Op::add(abar, Op::abs(nbar))));
    const T nhbM = Op::sub(Op::c(0.0f), hbM);
    auto row = [&](T fl, T fr, T jump, T corr) {
        return Op::fma(hbc, jump, Op::fma(nhbM, corr, Op::sub(Op::mul(hb1, fl), Op::mul(hb2, fr))));
    };
    const T rHl = Op::mul(L.rho, L.H), rHr = Op::mul(R.rho, R.H);
    out[0] = row(L.mn, R.mn, drho, delta1);
    out[1] = row(Op::fma(L.mn, L.n, L.p), Op::fma(R.mn, R.n, R.p), Op::sub(R.mn, L.mn), Op::mul(delta1, nbar));
    out[2] = row(Op::mul(L.mn, L.t), Op::mul(R.mn, R.t), Op::sub(R.mt, L.mt),
                 Op::fma(delta1, tbar, Op::mul(rhobar, Op::sub(R.t, L.t))));
    out[3] = row(Op::mul(rHl, L.n), Op::mul(rHr, R.n), Op::sub(rHr, rHl),
                 Op::fma(delta1, Hbar, Op::mul(rhobar, Op::sub(R.H, L.H))));
}

// A record [rho, u, v, p, H, sqrt(rho), rho u, rho v] as one side of a face
// with normal +x (DIR 0) or +y (DIR 1).
template <int DIR>
__device__ __forceinline__ AxisSide<float> axis_side(const float *P)
{
    return AxisSide<float>{P[0], P[DIR == 0 ? 1 : 2], P[DIR == 0 ? 2 : 1], P[3],
                           P[4], P[5], P[DIR == 0 ? 6 : 7], P[DIR == 0 ? 7 : 6]};
}

// The flux of an axis-aligned face with a positive normal of length h,
// direction known at compile time (DIR 0: n = (h,0), DIR 1: n = (0,h)).
template <int DIR>
__device__ __forceinline__ void roe_flux_axis_fp32(const float *L, const float *R, float h, float flux[4])
{
    float o[4];
    roe_flux_rot<LaneF1>(axis_side<DIR>(L), axis_side<DIR>(R), h, o);
    flux[0] = o[0];
    flux[DIR == 0 ? 1 : 2] = o[1];
    flux[DIR == 0 ? 2 : 1] = o[2];
    flux[3] = o[3];
}

// A cell's two interior faces at once in packed pairs: its x-face (low
// side Lx, normal +x, length hx_face) in the first half and its y-face (low
// side Ly, normal +y, length hy_face) in the second, both with high side P.
// Each half carries exactly the bits roe_flux_axis_fp32 gives that face.
__device__ __forceinline__ void roe_flux_axis_pair_fp32(const float *Lx, const float *Ly, const float *P,
                                                        float hx_face, float hy_face, float fx[4], float fy[4])
{
    const AxisSide<float> lx = axis_side<0>(Lx), ly = axis_side<1>(Ly), rx = axis_side<0>(P), ry = axis_side<1>(P);
    auto pair = [](const AxisSide<float> &a, const AxisSide<float> &b) {
        return AxisSide<float2>{make_float2(a.rho, b.rho), make_float2(a.n, b.n), make_float2(a.t, b.t),
                                make_float2(a.p, b.p),     make_float2(a.H, b.H), make_float2(a.sr, b.sr),
                                make_float2(a.mn, b.mn),   make_float2(a.mt, b.mt)};
    };
    float2 o[4];
    roe_flux_rot<LaneF2>(pair(lx, ly), pair(rx, ry), make_float2(hx_face, hy_face), o);
    fx[0] = o[0].x;
    fx[1] = o[1].x;
    fx[2] = o[2].x;
    fx[3] = o[3].x;
    fy[0] = o[0].y;
    fy[2] = o[1].y;
    fy[1] = o[2].y;
    fy[3] = o[3].y;
}

__device__ __forceinline__ void roe_flux_prim_fp32(const float *L, const float *R, float n0, float n1,
                                                   float flux[4])
{
    const bool xdir = (n1 == 0.0f);
    const bool ydir = (n0 == 0.0f);
    if (!(xdir || ydir)) {
        float ql[4] = {L[0], L[6], L[7], L[0] * L[4] - L[3]};
        float qr[4] = {R[0], R[6], R[7], R[0] * R[4] - R[3]};
        roe_flux_fp32(ql, qr, n0, n1, flux);
        return;
    }
    const float mag = xdir ? fabsf(n0) : fabsf(n1);
    const float sgn = xdir ? (n0 > 0.0f ? 1.0f : -1.0f) : (n1 > 0.0f ? 1.0f : -1.0f);
    const float rhol = L[0], ul = L[1], vl = L[2], pl = L[3], Hl = L[4], srl = L[5];
    const float rhor = R[0], ur = R[1], vr = R[2], pr = R[3], Hr = R[4], srr = R[5];
    // normal / tangential momentum components of each state
    const float unl = sgn * (xdir ? ul : vl), unr = sgn * (xdir ? ur : vr);
    const float inv = frcp(srl + srr);
    const float rhobar = srl * srr;
    const float ubar = (ul * srl + ur * srr) * inv;
    const float vbar = (vl * srl + vr * srr) * inv;
    const float Hbar = (Hl * srl + Hr * srr) * inv;
    const float a2 = 0.4f * (Hbar - 0.5f * (ubar * ubar + vbar * vbar));
    const float abar = sqrtf(a2);
    const float unbar = sgn * (xdir ? ubar : vbar);
    const float b1 = fmaxf(fmaxf(unbar + abar, unr + abar), 0.0f);
    const float b2 = fminf(fminf(unbar - abar, unl - abar), 0.0f);
    const float inv_db = frcp(b1 - b2);
    const float bcoeff = b1 * b2 * inv_db;
    const float delta1 = (rhor - rhol) - (pr - pl) * frcp(a2);
    const float bM = bcoeff * abar * frcp(abar + fabsf(unbar));
    // mass flux of each state through the face
    const float ml = sgn * (xdir ? L[6] : L[7]);
    const float mr = sgn * (xdir ? R[6] : R[7]);
    const float rHl = rhol * Hl, rHr = rhor * Hr;
    float fl, fr, d;
    fl = ml;
    fr = mr;
    d = bcoeff * (rhor - rhol) - bM * delta1;
    flux[0] = ((b1 * fl - b2 * fr) * inv_db + d) * mag;
    fl = ml * ul + (xdir ? sgn * pl : 0.0f);
    fr = mr * ur + (xdir ? sgn * pr : 0.0f);
    d = bcoeff * (R[6] - L[6]) - bM * (delta1 * ubar + (xdir ? 0.0f : rhobar * (ur - ul)));
    flux[1] = ((b1 * fl - b2 * fr) * inv_db + d) * mag;
    fl = ml * vl + (xdir ? 0.0f : sgn * pl);
    fr = mr * vr + (xdir ? 0.0f : sgn * pr);
    d = bcoeff * (R[7] - L[7]) - bM * (delta1 * vbar + (xdir ? rhobar * (vr - vl) : 0.0f));
    flux[2] = ((b1 * fl - b2 * fr) * inv_db + d) * mag;
    fl = rHl * unl;
    fr = rHr * unr;
    d = bcoeff * (rHr - rHl) - bM * (delta1 * Hbar + rhobar * (Hr - Hl));
    flux[3] = ((b1 * fl - b2 * fr) * inv_db + d) * mag;
}

// Boundary face on an FP32 record: conserved state rebuilt from the record.
__device__ __forceinline__ void bc_flux_rec_fp32(int bc, const float *P, float n0, float n1,
                                                 const float qin[4], float flux[4]);

__device__ __forceinline__ void bc_flux_fp32(int bc, const float q[4], float n0, float n1,
                                             const float qin[4], float flux[4])
{
    float qb[4];
    float oneOrho = frcp(q[0]);
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
    float oor = frcp(qb[0]);
    float ub = qb[1] * oor, vb = qb[2] * oor;
    float p = 0.4f * (qb[3] - 0.5f * qb[0] * (ub * ub + vb * vb));
    flux[0] = qb[1] * n0 + qb[2] * n1;
    flux[1] = (qb[1] * ub + p) * n0 + (qb[2] * ub) * n1;
    flux[2] = (qb[1] * vb) * n0 + (qb[2] * vb + p) * n1;
    flux[3] = (ub * n0 + vb * n1) * (qb[3] + p);
}

__device__ __forceinline__ void bc_flux_rec_fp32(int bc, const float *P, float n0, float n1,
                                                 const float qin[4], float flux[4])
{
    float q[4] = {P[0], P[6], P[7], P[0] * P[4] - P[3]};
    bc_flux_fp32(bc, q, n0, n1, qin, flux);
}

// One cell's CFL step candidate cfl*sqrt(volume)/(|V| + c) of
// solver_time_step_2d_module.F90:106-116, in FP32 with approximate square
// roots and reciprocals (the FP32-flux form; the state stays FP64).
__device__ __forceinline__ double cfl_candidate_fp32(const double q[4], double volume, double cfl)
{
    const float rho = (float)q[0];
    const float oneOrho = frcp(rho);
    const float u = (float)q[1] * oneOrho;
    const float v = (float)q[2] * oneOrho;
    const float V2 = u * u + v * v;
    const float pOverRho = 0.4f * ((float)q[3] * oneOrho - 0.5f * V2);
    const float eig = sqrtf(V2) + sqrtf(1.4f * pOverRho);
    return (double)((float)cfl * sqrtf((float)volume) * frcp(eig));
}

}  // namespace amrgpu
