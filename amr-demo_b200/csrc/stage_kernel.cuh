// stage_kernel.cuh -- one Runge-Kutta stage of the structured 2D residual,
// fused: neighbour-strip gather, face fluxes, residual assembly, division by
// the sub-cell volume, RK stage update, and (on the last stage of a step)
// the next step's CFL min-reduction and the L2 residual norm.
//
// It replaces, per stage, the reference's
//   physics_mpi_real_to_ghost  (physics_mpi.c:47-122; on one GPU the
//                               neighbour strips are read straight from HBM)
//   physics_rhs_structured     (physics_rhs_structured.c:19-283) with its
//     face kernels solver_residual_{bc,face_full,face_full_hang,
//     face_hang_full}_structured_2d and solver_residual_subgrid_2d
//   physics_norm_L2_residual   (physics_norm_residual.c:15-56)
//   the RK update loops of rk_1..lserk_45 (rk_time_integrators.c:22-540)
//   physics_time_step + MPI_Allreduce(MIN) (physics_time_step.c:16-49,
//     physics_runge_kutta_interface.c:197-205) for the following step.
//
// Work decomposition: a persistent grid; each CTA owns QPB quadrants at a
// time. Phase A stages the QPB patches (SoA, vectorised loads), the
// neighbour edge strips and the (n+1)^2 bilinear nodes in shared memory.
// Phase B evaluates every face flux of the patches once (interior faces
// first, then the 4n edge faces; a coarse quad's hanging edge evaluates two
// fluxes per edge cell). Phase C assembles each cell's residual in exactly
// the reference's accumulation order -- edge-face contributions in
// face_info order, then -F(x-1/2) +F(x+1/2) -F(y-1/2) +F(y+1/2) -- divides
// by the volume, negates, and applies the stage update. Edge fluxes are
// computed redundantly by both patches that share an edge, so there are no
// atomics and both sides see bit-identical values (conservation holds
// exactly as in the reference).
#pragma once

#include <cstdint>
#include <type_traits>

#include "device_common.cuh"

namespace amrgpu {

enum Scheme : int {
    kSchemeRhsOnly = 0,
    kSchemeRK1 = 1,
    kSchemeRK2 = 2,
    kSchemeRK3 = 3,
    kSchemeRK4 = 4,
    kSchemeLSERK45 = 5,
    kSchemeRK3ShuOsher = 6
};

struct StageArgs {
    const QuadDesc *quads;
    const double *qin;    // halo-read state, field f at qin + f*stride
    const double *a0;     // own-cell auxiliary inputs (same layout)
    const double *a1;
    double *out0;         // own-cell outputs
    double *out1;
    double *partials;     // one double per block
    DeviceScalars *scal;
    long long stride;     // field stride in doubles
    int nquad;            // quads updated (real quads)
    int scheme;
    int stage;            // 1-based
    int last_stage;       // 1: CFL for the next step, norm, time advance
    int cfl_on;           // 0: dt is the cap (the reference's RK2 path)
    int slot_read, slot_write, slot_reset;
    double h_base;        // coarse_grid_h
    double cfl;
    double dt_cap;
    double final_time;    // > 0: clip the step at this time
    double qinflow[4];    // bc 3 state (extension)
};

struct CflArgs {
    const QuadDesc *quads;
    const double *qin;
    DeviceScalars *scal;
    long long stride;
    int nquad;
    int slot;
    double cfl;
};

// LSERK45 coefficients, rk_time_integrators.c:439-448.
__device__ __forceinline__ void lserk_coeff(int stage, double &ra, double &rb)
{
    switch (stage) {
    case 1: ra = 0.0; rb = 1432997174477.0 / 9575080441755.0; break;
    case 2: ra = -567301805773.0 / 1357537059087.0; rb = 5161836677717.0 / 13612068292357.0; break;
    case 3: ra = -2404267990393.0 / 2016746695238.0; rb = 1720146321549.0 / 2090206949498.0; break;
    case 4: ra = -3550918686646.0 / 2091501179385.0; rb = 3134564353537.0 / 4481467310338.0; break;
    default: ra = -1275806237668.0 / 842570457699.0; rb = 2277821191437.0 / 14882151754819.0; break;
    }
}

// bilinear_node_2d_module.F90:14-36, left-to-right evaluation.
__device__ __forceinline__ void bilinear_node(const double *g, double xi, double eta, double &x,
                                              double &y)
{
    double oneMxi = 0.5 * (1.0 - xi);
    double onePxi = 0.5 * (1.0 + xi);
    double oneMeta = 0.5 * (1.0 - eta);
    double onePeta = 0.5 * (1.0 + eta);
    x = g[0] * oneMxi * oneMeta + g[2] * onePxi * oneMeta + g[4] * oneMxi * onePeta +
        g[6] * onePxi * onePeta;
    y = g[1] * oneMxi * oneMeta + g[3] * onePxi * oneMeta + g[5] * oneMxi * onePeta +
        g[7] * onePxi * onePeta;
}

// cell_h = h_base * (1/2**level) / n, e.g.
// solver_residual_face_full_structured_2d_module.F90:239
__device__ __forceinline__ double cell_h_of(double h_base, int level, int n)
{
    return h_base * (1.0 / ldexp(1.0, level)) / (double)n;
}

// Volume of the sub-cell with nodes a=n1, b=n2, c=n3, d=n4:
// 0.5*sqrt(((n4-n1) x (n3-n2))**2), solver_residual_subgrid_2d_module.F90:152-160
__device__ __forceinline__ double subcell_volume(double x1, double y1, double x2, double y2,
                                                 double x3, double y3, double x4, double y4)
{
    double v1x = x4 - x1, v1y = y4 - y1;
    double v2x = x3 - x2, v2y = y3 - y2;
    double cr = v1x * v2y - v1y * v2x;
    return 0.5 * sqrt(cr * cr);
}

__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = (w < v) ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Shared-memory footprint of one stage CTA.
template <int N, int QPB, bool F32>
struct StageSmem {
    using R = typename std::conditional<F32, float, double>::type;
    static constexpr int NN = N * N;
    static constexpr int NP1 = N + 1;
    static constexpr size_t desc = sizeof(QuadDesc) * QPB;
    static constexpr size_t qs = sizeof(double) * QPB * 4 * NN;
    static constexpr size_t qf = F32 ? sizeof(float) * QPB * 4 * NN : 0;
    static constexpr size_t strip = sizeof(R) * QPB * 4 * 2 * 4 * N;
    static constexpr size_t nodes = sizeof(double) * QPB * NP1 * NP1 * 2;
    static constexpr size_t fx = sizeof(R) * QPB * 4 * N * NP1;
    static constexpr size_t fy = sizeof(R) * QPB * 4 * NP1 * N;
    static constexpr size_t fh = sizeof(R) * QPB * 4 * 4 * N;
    static constexpr size_t red = sizeof(double) * 64;
    static constexpr size_t total = desc + qs + qf + strip + nodes + fx + fy + fh + red;
};

template <int N, int QPB, int T, int MINB, bool F32, typename FluxOps>
__global__ void __launch_bounds__(T, MINB) stage_kernel(const StageArgs a)
{
    using R = typename std::conditional<F32, float, double>::type;
    using S = StageSmem<N, QPB, F32>;
    constexpr int NN = N * N;
    constexpr int NP1 = N + 1;
    constexpr int NINT = 2 * N * (N - 1);   // interior faces per quad
    constexpr int NEDGE = 4 * N;            // edge faces per quad
    constexpr int NWORK = NINT + NEDGE;

    extern __shared__ __align__(16) unsigned char smem[];
    QuadDesc *sq = reinterpret_cast<QuadDesc *>(smem);
    double *qs = reinterpret_cast<double *>(smem + S::desc);
    R *qf = F32 ? reinterpret_cast<R *>(smem + S::desc + S::qs) : reinterpret_cast<R *>(qs);
    R *strip = reinterpret_cast<R *>(smem + S::desc + S::qs + S::qf);
    double *nodes = reinterpret_cast<double *>(smem + S::desc + S::qs + S::qf + S::strip);
    R *fx = reinterpret_cast<R *>(smem + S::desc + S::qs + S::qf + S::strip + S::nodes);
    R *fy = fx + QPB * 4 * N * NP1;
    R *fh = fy + QPB * 4 * NP1 * N;
    double *red = reinterpret_cast<double *>(smem + S::total - S::red);

    const int tid = threadIdx.x;
    const long long stride = a.stride;
    const double scale_factor = 2.0 / (double)N;

    // step scalars
    const StepSlot slot = a.scal->slot[a.slot_read];
    double dt = __longlong_as_double((long long)slot.dt_bits);
    if (!a.cfl_on) dt = a.dt_cap;
    if (a.final_time > 0.0) {
        double rem = a.final_time - slot.time;
        if (rem < dt) dt = rem;
        if (dt < 0.0) dt = 0.0;
    }
    if (a.last_stage && blockIdx.x == 0 && tid == 0) {
        a.scal->slot[a.slot_write].time = slot.time + dt;
        a.scal->dt_used = dt;
        if (dt > 0.0) a.scal->steps += 1;
        a.scal->slot[a.slot_reset].dt_bits = (unsigned long long)__double_as_longlong(a.dt_cap);
        if (!a.cfl_on) a.scal->slot[a.slot_write].dt_bits = (unsigned long long)__double_as_longlong(a.dt_cap);
    }

    double my_dt_min = a.dt_cap;
    double my_norm = 0.0;
    int my_flags = 0;

    for (int grp = blockIdx.x; grp * QPB < a.nquad; grp += gridDim.x) {
        const int q0 = grp * QPB;
        // ---------------- phase A: descriptors, patches, strips, nodes
        {
            const int *src = reinterpret_cast<const int *>(a.quads + q0);
            int *dst = reinterpret_cast<int *>(sq);
            constexpr int per = sizeof(QuadDesc) / 4;
            const int lim = min(QPB, a.nquad - q0) * per;
            for (int k = tid; k < lim; k += T) dst[k] = __ldg(src + k);
        }
        {
            constexpr int H = NN / 2;  // double2 per field slab
            for (int k = tid; k < QPB * 4 * H; k += T) {
                int ql = k / (4 * H);
                int rem = k - ql * 4 * H;
                int f = rem / H;
                int c2 = rem - f * H;
                if (q0 + ql < a.nquad) {
                    const double2 v = __ldg(reinterpret_cast<const double2 *>(
                        a.qin + f * stride + (long long)(q0 + ql) * NN) + c2);
                    double *d = qs + (ql * 4 + f) * NN + 2 * c2;
                    d[0] = v.x;
                    d[1] = v.y;
                    if (F32) {
                        qf[(ql * 4 + f) * NN + 2 * c2] = (R)v.x;
                        qf[(ql * 4 + f) * NN + 2 * c2 + 1] = (R)v.y;
                    }
                }
            }
        }
        __syncthreads();
        // neighbour edge strips: [ql][side][k][f][m]
        for (int k = tid; k < QPB * 4 * 2 * 4 * N; k += T) {
            int m = k % N;
            int f = (k / N) % 4;
            int kk = (k / (4 * N)) % 2;
            int s = (k / (8 * N)) % 4;
            int ql = k / (32 * N);
            if (q0 + ql >= a.nquad) continue;
            const SideDesc &d = sq[ql].side[s];
            int nbr = -1;
            if (d.kind == kSideFull || d.kind == kSideFineHang) nbr = (kk == 0) ? d.nbr0 : -1;
            else if (d.kind == kSideCoarseHang) nbr = (kk == 0) ? d.nbr0 : d.nbr1;
            if (nbr < 0) continue;
            // the neighbour's edge facing this side
            int ci, cj;
            if (s == 0) { ci = N - 1; cj = m; }
            else if (s == 1) { ci = 0; cj = m; }
            else if (s == 2) { ci = m; cj = N - 1; }
            else { ci = m; cj = 0; }
            strip[k] = (R)__ldg(a.qin + f * stride + (long long)nbr * NN + cj * N + ci);
        }
        // bilinear nodes N(k,l) = map(s*k - 1, s*l - 1)
        for (int k = tid; k < QPB * NP1 * NP1; k += T) {
            int ql = k / (NP1 * NP1);
            int r = k - ql * NP1 * NP1;
            int l = r / NP1;
            int kx = r - l * NP1;
            if (q0 + ql >= a.nquad) continue;
            double x, y;
            bilinear_node(sq[ql].corner, scale_factor * (double)kx - 1.0,
                          scale_factor * (double)l - 1.0, x, y);
            nodes[2 * k] = x;
            nodes[2 * k + 1] = y;
        }
        __syncthreads();

        // ---------------- phase B: face fluxes
        for (int k = tid; k < QPB * NWORK; k += T) {
            int ql, r;
            if (k < QPB * NINT) { ql = k / NINT; r = k - ql * NINT; }
            else { int e = k - QPB * NINT; ql = e / NEDGE; r = NINT + (e - ql * NEDGE); }
            if (q0 + ql >= a.nquad) continue;
            const R *qp = qf + ql * 4 * NN;
            const double *nd = nodes + ql * NP1 * NP1 * 2;
            R q_l[4], q_r[4], fl[4];
            if (r < N * (N - 1)) {
                // interior x-face between cells (ax-1, j) and (ax, j)
                int j = r / (N - 1);
                int ax = 1 + (r - j * (N - 1));
                const double *p1 = nd + 2 * (j * NP1 + ax);
                const double *p2 = nd + 2 * ((j + 1) * NP1 + ax);
                R n0 = (R)(p2[1] - p1[1]);
                R n1 = (R)(p1[0] - p2[0]);
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    q_l[f] = qp[f * NN + j * N + ax - 1];
                    q_r[f] = qp[f * NN + j * N + ax];
                }
                FluxOps::roe(q_l, q_r, n0, n1, fl);
#pragma unroll
                for (int f = 0; f < 4; ++f) fx[((ql * 4 + f) * N + j) * NP1 + ax] = fl[f];
            } else if (r < NINT) {
                // interior y-face between cells (i, ay-1) and (i, ay)
                int r2 = r - N * (N - 1);
                int ay = 1 + r2 / N;
                int i = r2 - (ay - 1) * N;
                const double *p1 = nd + 2 * (ay * NP1 + i + 1);
                const double *p2 = nd + 2 * (ay * NP1 + i);
                R n0 = (R)(p2[1] - p1[1]);
                R n1 = (R)(p1[0] - p2[0]);
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    q_l[f] = qp[f * NN + (ay - 1) * N + i];
                    q_r[f] = qp[f * NN + ay * N + i];
                }
                FluxOps::roe(q_l, q_r, n0, n1, fl);
#pragma unroll
                for (int f = 0; f < 4; ++f) fy[((ql * 4 + f) * NP1 + ay) * N + i] = fl[f];
            } else {
                // edge face of side s at position m
                int e = r - NINT;
                int s = e / N;
                int m = e - s * N;
                const SideDesc &d = sq[ql].side[s];
                int ci = (s == 0) ? 0 : (s == 1) ? N - 1 : m;
                int cj = (s == 2) ? 0 : (s == 3) ? N - 1 : m;
                R own[4];
#pragma unroll
                for (int f = 0; f < 4; ++f) own[f] = qp[f * NN + cj * N + ci];
                double ch = cell_h_of(a.h_base, d.level, N);
                R h = (R)ch;
                R n0 = (s < 2) ? h : (R)0;
                R n1 = (s < 2) ? (R)0 : h;
                if (d.kind == kSideBoundary) {
                    if (s == 0) n0 = -h;
                    if (s == 2) n1 = -h;
                    R qin[4] = {(R)a.qinflow[0], (R)a.qinflow[1], (R)a.qinflow[2], (R)a.qinflow[3]};
                    FluxOps::bc(d.bc, own, n0, n1, qin, fl);
                } else {
                    const R *sp = strip + ((ql * 4 + s) * 2) * 4 * N;
                    R nb[4];
#pragma unroll
                    for (int f = 0; f < 4; ++f) nb[f] = sp[f * N + m];
                    if (s & 1) FluxOps::roe(own, nb, n0, n1, fl);
                    else FluxOps::roe(nb, own, n0, n1, fl);
                    if (d.kind == kSideCoarseHang) {
                        R fl2[4];
#pragma unroll
                        for (int f = 0; f < 4; ++f) nb[f] = sp[4 * N + f * N + m];
                        if (s & 1) FluxOps::roe(own, nb, n0, n1, fl2);
                        else FluxOps::roe(nb, own, n0, n1, fl2);
#pragma unroll
                        for (int f = 0; f < 4; ++f) fh[((ql * 4 + s) * 4 + f) * N + m] = fl2[f];
                    }
                }
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    if (s < 2) fx[((ql * 4 + f) * N + m) * NP1 + (s == 0 ? 0 : N)] = fl[f];
                    else fy[((ql * 4 + f) * NP1 + (s == 2 ? 0 : N)) * N + m] = fl[f];
                }
            }
        }
        __syncthreads();

        // ---------------- phase C: residual assembly and stage update
        for (int k = tid; k < QPB * NN; k += T) {
            int ql = k / NN;
            int c = k - ql * NN;
            if (q0 + ql >= a.nquad) continue;
            int i = c % N, j = c / N;
            const QuadDesc &qd = sq[ql];
            double r[4] = {0.0, 0.0, 0.0, 0.0};
            int sx = (i == 0) ? 0 : (i == N - 1) ? 1 : -1;
            int sy = (j == 0) ? 2 : (j == N - 1) ? 3 : -1;
            int first = sx, second = sy;
            if (sx >= 0 && sy >= 0 && qd.side[sy].rank < qd.side[sx].rank) { first = sy; second = sx; }
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                int s = pass == 0 ? first : second;
                if (s < 0) continue;
                int kind = qd.side[s].kind;
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    double F = (s < 2) ? (double)fx[((ql * 4 + f) * N + j) * NP1 + (s == 0 ? 0 : N)]
                                       : (double)fy[((ql * 4 + f) * NP1 + (s == 2 ? 0 : N)) * N + i];
                    int m = (s < 2) ? j : i;
                    if (kind == kSideBoundary || (s & 1)) {
                        r[f] = r[f] + F;
                        if (kind == kSideCoarseHang) r[f] = r[f] + (double)fh[((ql * 4 + s) * 4 + f) * N + m];
                    } else {
                        r[f] = r[f] - F;
                        if (kind == kSideCoarseHang) r[f] = r[f] - (double)fh[((ql * 4 + s) * 4 + f) * N + m];
                    }
                }
            }
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                if (i > 0) r[f] = r[f] - (double)fx[((ql * 4 + f) * N + j) * NP1 + i];
                if (i < N - 1) r[f] = r[f] + (double)fx[((ql * 4 + f) * N + j) * NP1 + i + 1];
            }
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                if (j > 0) r[f] = r[f] - (double)fy[((ql * 4 + f) * NP1 + j) * N + i];
                if (j < N - 1) r[f] = r[f] + (double)fy[((ql * 4 + f) * NP1 + j + 1) * N + i];
            }
            const double *nd = nodes + ql * NP1 * NP1 * 2;
            const double *n1p = nd + 2 * (j * NP1 + i);
            const double *n3p = nd + 2 * ((j + 1) * NP1 + i);
            double vol = subcell_volume(n1p[0], n1p[1], n1p[2], n1p[3], n3p[0], n3p[1], n3p[2], n3p[3]);
            double kv[4];
            if (F32) {
                double inv = 1.0 / vol;
#pragma unroll
                for (int f = 0; f < 4; ++f) kv[f] = -(r[f] * inv);
            } else {
#pragma unroll
                for (int f = 0; f < 4; ++f) kv[f] = (r[f] / vol) * -1.0;
            }

            const long long gi = (long long)(q0 + ql) * NN + c;
            double q0v[4], qn[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) q0v[f] = qs[(ql * 4 + f) * NN + c];

            switch (a.scheme) {
            case kSchemeRhsOnly:
#pragma unroll
                for (int f = 0; f < 4; ++f) { a.out0[f * stride + gi] = kv[f]; qn[f] = q0v[f]; }
                break;
            case kSchemeRK1: {
                double beta1 = 1.0 * dt;
#pragma unroll
                for (int f = 0; f < 4; ++f) { qn[f] = q0v[f] + beta1 * kv[f]; a.out0[f * stride + gi] = qn[f]; }
                break;
            }
            case kSchemeRK2: {
                double alpha1 = 1.0 * dt, beta1 = 0.5 * dt, beta2 = 0.5 * dt;
                if (a.stage == 1) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        qn[f] = q0v[f] + alpha1 * kv[f];
                        a.out0[f * stride + gi] = qn[f];
                        a.out1[f * stride + gi] = q0v[f] + beta1 * kv[f];
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        qn[f] = a.a0[f * stride + gi] + beta2 * kv[f];
                        a.out0[f * stride + gi] = qn[f];
                    }
                }
                break;
            }
            case kSchemeRK3: {
                double alpha1 = 1.00 * dt, alpha21 = 0.25 * dt, alpha22 = 0.25 * dt;
                double beta1 = 1.0 / 6.0 * dt, beta2 = 1.0 / 6.0 * dt, beta3 = 2.0 / 3.0 * dt;
                if (a.stage == 1) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        qn[f] = q0v[f] + alpha1 * kv[f];
                        a.out0[f * stride + gi] = qn[f];
                        a.out1[f * stride + gi] = kv[f];
                    }
                } else if (a.stage == 2) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        double Q0 = a.a0[f * stride + gi];
                        double k1 = a.a1[f * stride + gi];
                        qn[f] = Q0 + alpha21 * k1 + alpha22 * kv[f];
                        double C = Q0 + beta1 * k1 + beta2 * kv[f];
                        a.out0[f * stride + gi] = qn[f];
                        a.out1[f * stride + gi] = C;
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        qn[f] = a.a0[f * stride + gi] + beta3 * kv[f];
                        a.out0[f * stride + gi] = qn[f];
                    }
                }
                break;
            }
            case kSchemeRK4: {
                double alpha1 = 0.5 * dt, alpha2 = 0.5 * dt, alpha3 = 1.0 * dt, beta1 = 1.0 / 6.0 * dt;
                if (a.stage == 1) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        qn[f] = q0v[f] + alpha1 * kv[f];
                        a.out0[f * stride + gi] = qn[f];
                        a.out1[f * stride + gi] = kv[f];
                    }
                } else if (a.stage < 4) {
                    double al = (a.stage == 2) ? alpha2 : alpha3;
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        double Q0 = a.a0[f * stride + gi];
                        double K = a.a1[f * stride + gi];
                        qn[f] = Q0 + al * kv[f];
                        a.out0[f * stride + gi] = qn[f];
                        a.out1[f * stride + gi] = K + 2.0 * kv[f];
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        double Q0 = a.a0[f * stride + gi];
                        double K = a.a1[f * stride + gi];
                        qn[f] = Q0 + beta1 * (K + kv[f]);
                        a.out0[f * stride + gi] = qn[f];
                    }
                }
                break;
            }
            case kSchemeLSERK45: {
                double ra, rb;
                lserk_coeff(a.stage, ra, rb);
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    double qsv = (a.stage == 1) ? dt * kv[f] : a.a0[f * stride + gi] * ra + dt * kv[f];
                    qn[f] = q0v[f] + rb * qsv;
                    a.out1[f * stride + gi] = qsv;
                    a.out0[f * stride + gi] = qn[f];
                }
                break;
            }
            default: {  // kSchemeRK3ShuOsher
                if (a.stage == 1) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) { qn[f] = q0v[f] + dt * kv[f]; a.out0[f * stride + gi] = qn[f]; }
                } else if (a.stage == 2) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        qn[f] = 0.75 * a.a0[f * stride + gi] + 0.25 * (q0v[f] + dt * kv[f]);
                        a.out0[f * stride + gi] = qn[f];
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        qn[f] = (1.0 / 3.0) * a.a0[f * stride + gi] + (2.0 / 3.0) * (q0v[f] + dt * kv[f]);
                        a.out0[f * stride + gi] = qn[f];
                    }
                }
                break;
            }
            }

            if (a.last_stage) {
#pragma unroll
                for (int f = 0; f < 4; ++f) my_norm += kv[f] * kv[f];
                if (a.cfl_on) {
                    double cand = FluxOps::cfl(qn, vol, a.cfl);
                    if (cand < my_dt_min) my_dt_min = cand;
                }
                double rho = qn[0];
                double pe = qn[3] - 0.5 * (qn[1] * qn[1] + qn[2] * qn[2]) / rho;
                if (!(rho > 0.0) || !(pe > 0.0)) my_flags |= kFlagNegative;
            }
        }
        __syncthreads();
    }

    if (!a.last_stage) return;

    // ---------------- block reductions: CFL min (one atomic per block) and
    // the residual norm (per-block partials, summed in block order by the
    // last block to finish, so the result does not depend on scheduling).
    const int lane = tid & 31, warp = tid >> 5;
    double wmin = warp_min(my_dt_min);
    double wsum = warp_sum(my_norm);
    int wflags = __reduce_or_sync(0xffffffffu, my_flags);
    if (lane == 0) { red[warp] = wmin; red[32 + warp] = wsum; }
    if (wflags && lane == 0) atomicOr(&a.scal->flags, wflags);
    __syncthreads();
    if (tid == 0) {
        double bmin = red[0], bsum = red[32];
        for (int w = 1; w < T / 32; ++w) {
            bmin = (red[w] < bmin) ? red[w] : bmin;
            bsum += red[32 + w];
        }
        if (a.cfl_on)
            atomicMin(&a.scal->slot[a.slot_write].dt_bits, (unsigned long long)__double_as_longlong(bmin));
        a.partials[blockIdx.x] = bsum;
        __threadfence();
        unsigned ticket = atomicAdd(&a.scal->done_blocks, 1u);
        if (ticket == gridDim.x - 1) {
            __threadfence();
            double tot = 0.0;
            for (int b = 0; b < (int)gridDim.x; ++b) tot += ((volatile double *)a.partials)[b];
            a.scal->norm_sq = tot;
            if (!isfinite(tot)) atomicOr(&a.scal->flags, kFlagNonFinite);
            a.scal->done_blocks = 0u;
        }
    }
}

}  // namespace amrgpu
