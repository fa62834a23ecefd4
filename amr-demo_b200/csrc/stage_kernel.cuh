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
// time and walks its groups in a software pipeline. While group k is being
// computed, group k+1's four field slabs per quad (contiguous n*n doubles
// each) arrive through 1D bulk copies (TMA engine) completed on an
// mbarrier, its neighbour edge strips through cp.async, and group k+2's
// descriptors through a bulk copy; the FP32 form's first own-cell auxiliary
// input comes with the slabs, the other auxiliary arrays are prefetched into
// L2.
//   A  per-cell primitive records (rho, rho*u, rho*v, rho*E, u, v, p, H,
//      sqrt(rho)) of the patches and strips, and the (n+1)^2 bilinear nodes
//   B  every face flux once (interior faces first, then the 4n edge faces;
//      a coarse quad's hanging edge evaluates two fluxes per edge cell)
//   C  each cell's residual -- in the FP64 form in exactly the reference's
//      accumulation order (edge-face contributions in face_info order, then
//      -F(x-1/2) +F(x+1/2) -F(y-1/2) +F(y+1/2)); in the FP32 form the four
//      faces alike, edges included, plus a coarse hanging edge's second flux
//      -- divided by the volume, negated, and the stage update.
// Edge fluxes are computed by both patches that share an edge, so there are
// no atomics and both sides see bit-identical values; conservation holds
// exactly as in the reference.
#pragma once

#include <cstdint>
#include <type_traits>

#include "async_copy.cuh"
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
    // mixed patch sizes: per-quad sizes and offsets, and the work list
    // (the 16x16 quads first, nwork16 of them, then the 8x8 quads in pairs,
    // nwork8 of them)
    const MixDesc *mix;
    const int *work;
    int nwork16;
    int nwork8;
};

struct CflArgs {
    const QuadDesc *quads;
    const MixDesc *mix;  // mixed patch sizes: per-quad n and offset (else null)
    const double *qin;
    DeviceScalars *scal;
    long long stride;
    int nquad;
    int slot;
    double cfl;
};

// Arguments of remap_cfl_kernel (remap_cfl.cuh): the remap's old state,
// kind and source per new quad, and the CFL prologue's arguments for the
// new mesh (cfl.qin unused; cfl.stride is the new state's field stride).
struct RemapCflArgs {
    const double *qold;
    long long stride_old;
    double *qnew;
    const int *kind;
    const int *src;
    CflArgs cfl;
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
    // h_base / 2^level / n with n a power of two: both steps scale by a power
    // of two and are exact, so two multiplications by exact powers of two
    // (built from their exponent bits) give the same value as the divisions
    // without the IEEE division sequences; level and n stay far inside the
    // normal exponent range
    const double inv_2l = __longlong_as_double((long long)(1023 - level) << 52);
    const double inv_n = __longlong_as_double((long long)(1023 - (__ffs(n) - 1)) << 52);
    return h_base * inv_2l * inv_n;
}

// Volume of the sub-cell with nodes n1..n4:
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

constexpr unsigned kWaitLimit = 1u << 22;  // bounded mbarrier polls

// Per-cell records and per-face fluxes are stored array-of-structures in
// shared memory so each is moved with 16-byte vector accesses:
//   FP32 record: 8 floats (2 x float4), flux: float4
//   FP64 record: 10 doubles (5 x double2, slot 9 unused), flux: 2 x double2
template <bool F32>
struct RecTraits;
template <>
struct RecTraits<true> {
    using R = float;
    using V = float4;
    static constexpr int n = 8;
    static constexpr int nv = 2;
    static constexpr int fv = 1;  // vectors per flux
};
template <>
struct RecTraits<false> {
    using R = double;
    using V = double2;
    static constexpr int n = 10;
    static constexpr int nv = 5;
    static constexpr int fv = 2;
};

template <bool F32>
__device__ __forceinline__ void load_rec(const typename RecTraits<F32>::R *base, int idx,
                                         typename RecTraits<F32>::R *out)
{
    using T = RecTraits<F32>;
    const typename T::V *src = reinterpret_cast<const typename T::V *>(base + (size_t)idx * T::n);
    typename T::V *dst = reinterpret_cast<typename T::V *>(out);
#pragma unroll
    for (int k = 0; k < T::nv; ++k) dst[k] = src[k];
}

template <bool F32>
__device__ __forceinline__ void store_flux(typename RecTraits<F32>::R *base, int idx,
                                           const typename RecTraits<F32>::R *f)
{
    using T = RecTraits<F32>;
    typename T::V *dst = reinterpret_cast<typename T::V *>(base + (size_t)idx * 4);
    const typename T::V *src = reinterpret_cast<const typename T::V *>(f);
#pragma unroll
    for (int k = 0; k < T::fv; ++k) dst[k] = src[k];
}

template <bool F32>
__device__ __forceinline__ void load_flux(const typename RecTraits<F32>::R *base, int idx, double out[4])
{
    using T = RecTraits<F32>;
    alignas(16) typename T::R f[4];
    const typename T::V *src = reinterpret_cast<const typename T::V *>(base + (size_t)idx * 4);
    typename T::V *dst = reinterpret_cast<typename T::V *>(f);
#pragma unroll
    for (int k = 0; k < T::fv; ++k) dst[k] = src[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = (double)f[k];
}

// Shared-memory carve-up of one stage CTA (all offsets 16-byte aligned).
template <int N, int QPB, bool F32>
struct StageSmem {
    using R = typename RecTraits<F32>::R;
    static constexpr int NN = N * N;
    static constexpr int NP1 = N + 1;
    static constexpr int NSTRIP = 4 * 2 * N;        // strip cells per quad: side x {nbr0,nbr1} x m
    static constexpr int NPC = NN + NSTRIP;         // record cells per quad
    static constexpr size_t al(size_t b) { return (b + 15) / 16 * 16; }
    static constexpr size_t bar = 32;
    static constexpr size_t desc = al(sizeof(QuadDesc) * QPB) * 3;
    static constexpr size_t raw = al(sizeof(double) * QPB * 4 * NN) * 2;
    // FP32 form: the stage's first own-cell auxiliary input (Q0 of the
    // Shu-Osher stages) arrives with the slabs, double-buffered
    static constexpr size_t aux = F32 ? al(sizeof(double) * QPB * 4 * NN) * 2 : 0;
    static constexpr size_t rstrip = al(sizeof(double) * QPB * 4 * NSTRIP) * 2;
    static constexpr size_t prim = al(sizeof(R) * QPB * RecTraits<F32>::n * NPC);
    static constexpr size_t nodes = F32 ? 0 : al(sizeof(double) * QPB * NP1 * NP1 * 2);
    // per quad: hx, hy, 1/vol, vol (FP32 form), cell_h of sides 0..3
    static constexpr size_t geo = al(sizeof(double) * QPB * 8);
    static constexpr size_t fx = al(sizeof(R) * QPB * 4 * N * NP1);
    static constexpr size_t fy = al(sizeof(R) * QPB * 4 * NP1 * N);
    static constexpr size_t fh = al(sizeof(R) * QPB * 4 * 4 * N);
    static constexpr size_t red = sizeof(double) * 64;
    static constexpr size_t o_desc = bar;
    static constexpr size_t o_raw = o_desc + desc;
    static constexpr size_t o_aux = o_raw + raw;
    static constexpr size_t o_rstrip = o_aux + aux;
    static constexpr size_t o_prim = o_rstrip + rstrip;
    static constexpr size_t o_nodes = o_prim + prim;
    static constexpr size_t o_geo = o_nodes + nodes;
    static constexpr size_t o_fx = o_geo + geo;
    static constexpr size_t o_fy = o_fx + fx;
    static constexpr size_t o_fh = o_fy + fy;
    static constexpr size_t o_red = o_fh + fh;
    static constexpr size_t total = o_red + red;
};

// The neighbour's cell facing side s at position m (its opposite edge).
template <int N>
__device__ __forceinline__ int facing_cell(int s, int m)
{
    if (s == 0) return m * N + (N - 1);
    if (s == 1) return m * N;
    if (s == 2) return (N - 1) * N + m;
    return m;
}

// The stage update of one cell for every scheme, with the reference's
// coefficients and summation order (rk_time_integrators.c:22-540; the
// Shu-Osher RK3 of the FP32-flux form is the extension). kv is the cell's
// residual, q0v its input state, A0(f) / A1(f) the first / second auxiliary
// inputs; writes the outputs at gi and returns the new state in qn.
// SCHEME / STAGE >= 0 / > 0 fix the scheme and the stage at compile time
// (the same expressions, without the per-cell switch); -1 / 0 read them
// from the arguments.
template <int SCHEME = -1, int STAGE = 0, typename A0F, typename A1F>
__device__ __forceinline__ void rk_update(const StageArgs &a, double dt, long long stride, long long gi,
                                          const double q0v[4], const double kv[4], A0F A0, A1F A1, double qn[4])
{
    const int scheme = SCHEME >= 0 ? SCHEME : a.scheme;
    const int stage = STAGE > 0 ? STAGE : a.stage;
    switch (scheme) {
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
        if (stage == 1) {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                qn[f] = q0v[f] + alpha1 * kv[f];
                a.out0[f * stride + gi] = qn[f];
                a.out1[f * stride + gi] = q0v[f] + beta1 * kv[f];
            }
        } else {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                qn[f] = A0(f) + beta2 * kv[f];
                a.out0[f * stride + gi] = qn[f];
            }
        }
        break;
    }
    case kSchemeRK3: {
        double alpha1 = 1.00 * dt, alpha21 = 0.25 * dt, alpha22 = 0.25 * dt;
        double beta1 = 1.0 / 6.0 * dt, beta2 = 1.0 / 6.0 * dt, beta3 = 2.0 / 3.0 * dt;
        if (stage == 1) {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                qn[f] = q0v[f] + alpha1 * kv[f];
                a.out0[f * stride + gi] = qn[f];
                a.out1[f * stride + gi] = kv[f];
            }
        } else if (stage == 2) {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                double Q0 = A0(f);
                double k1 = A1(f);
                qn[f] = Q0 + alpha21 * k1 + alpha22 * kv[f];
                double C = Q0 + beta1 * k1 + beta2 * kv[f];
                a.out0[f * stride + gi] = qn[f];
                a.out1[f * stride + gi] = C;
            }
        } else {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                qn[f] = A0(f) + beta3 * kv[f];
                a.out0[f * stride + gi] = qn[f];
            }
        }
        break;
    }
    case kSchemeRK4: {
        double alpha1 = 0.5 * dt, alpha2 = 0.5 * dt, alpha3 = 1.0 * dt, beta1 = 1.0 / 6.0 * dt;
        if (stage == 1) {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                qn[f] = q0v[f] + alpha1 * kv[f];
                a.out0[f * stride + gi] = qn[f];
                a.out1[f * stride + gi] = kv[f];
            }
        } else if (stage < 4) {
            double al = (stage == 2) ? alpha2 : alpha3;
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                double Q0 = A0(f);
                double K = A1(f);
                qn[f] = Q0 + al * kv[f];
                a.out0[f * stride + gi] = qn[f];
                a.out1[f * stride + gi] = K + 2.0 * kv[f];
            }
        } else {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                double Q0 = A0(f);
                double K = A1(f);
                qn[f] = Q0 + beta1 * (K + kv[f]);
                a.out0[f * stride + gi] = qn[f];
            }
        }
        break;
    }
    case kSchemeLSERK45: {
        double ra, rb;
        lserk_coeff(stage, ra, rb);
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            double qsv = (stage == 1) ? dt * kv[f] : A0(f) * ra + dt * kv[f];
            qn[f] = q0v[f] + rb * qsv;
            a.out1[f * stride + gi] = qsv;
            a.out0[f * stride + gi] = qn[f];
        }
        break;
    }
    default: {  // kSchemeRK3ShuOsher
        if (stage == 1) {
#pragma unroll
            for (int f = 0; f < 4; ++f) { qn[f] = q0v[f] + dt * kv[f]; a.out0[f * stride + gi] = qn[f]; }
        } else if (stage == 2) {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                qn[f] = 0.75 * A0(f) + 0.25 * (q0v[f] + dt * kv[f]);
                a.out0[f * stride + gi] = qn[f];
            }
        } else {
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                qn[f] = (1.0 / 3.0) * A0(f) + (2.0 / 3.0) * (q0v[f] + dt * kv[f]);
                a.out0[f * stride + gi] = qn[f];
            }
        }
        break;
    }
    }
}

template <int N, int QPB, int T, int MINB, bool F32, typename FluxOps>
__global__ void __launch_bounds__(T, MINB) stage_kernel(const StageArgs a)
{
    using Tr = RecTraits<F32>;
    using R = typename Tr::R;
    using S = StageSmem<N, QPB, F32>;
    constexpr int RS = Tr::n;
    constexpr int NN = N * N;
    constexpr int NP1 = N + 1;
    constexpr int NPC = S::NPC;
    constexpr int NFACE = 2 * N * NP1;      // faces per quad (x and y, edges included)
    constexpr int RB = (QPB * NFACE + T - 1) / T;   // face rounds per thread
    static_assert(T % 32 == 0, "whole warps");
    static_assert(N <= 32 && QPB <= 64, "face code packing");

    stage_launch_gate();
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    QuadDesc *sdesc = reinterpret_cast<QuadDesc *>(smem + S::o_desc);
    double *sraw = reinterpret_cast<double *>(smem + S::o_raw);
    double *saux = reinterpret_cast<double *>(smem + S::o_aux);
    double *srstrip = reinterpret_cast<double *>(smem + S::o_rstrip);
    R *prim = reinterpret_cast<R *>(smem + S::o_prim);
    double *nodes = reinterpret_cast<double *>(smem + S::o_nodes);
    double *geo = reinterpret_cast<double *>(smem + S::o_geo);
    R *fx = reinterpret_cast<R *>(smem + S::o_fx);
    R *fy = reinterpret_cast<R *>(smem + S::o_fy);
    R *fh = reinterpret_cast<R *>(smem + S::o_fh);
    double *red = reinterpret_cast<double *>(smem + S::o_red);
    constexpr size_t desc_slot = S::desc / 3 / sizeof(QuadDesc);   // QuadDesc entries per slot
    constexpr size_t raw_slot = S::raw / 2 / sizeof(double);
    constexpr size_t aux_slot = S::aux / 2 / sizeof(double);
    const bool stage_a0 = F32 && a.a0 != nullptr;
    constexpr size_t rstrip_slot = S::rstrip / 2 / sizeof(double);

    const int tid = threadIdx.x;
    const long long stride = a.stride;
    const double scale_factor = 2.0 / (double)N;
    const int ngroups = (a.nquad + QPB - 1) / QPB;

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
        if (!a.cfl_on)
            a.scal->slot[a.slot_write].dt_bits = (unsigned long long)__double_as_longlong(a.dt_cap);
    }

    double my_dt_min = a.dt_cap;
    double my_norm = 0.0;
    int my_flags = 0;

    // Each thread's face work items are the same for every quad group:
    // decode them once. code = ql | xd<<6 | fa<<7 | fb<<13 | valid<<19.
    int fcode[RB];
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
        const int k = tid + rb * T;
        if (k < QPB * NFACE) {
            const int ql = k / NFACE;
            const int r = k - ql * NFACE;
            const int xd = r < N * NP1;
            int fa, fb;
            if (xd) { fb = r / NP1; fa = r - fb * NP1; }
            else { const int r2 = r - N * NP1; fa = r2 / N; fb = r2 - fa * N; }
            fcode[rb] = ql | (xd << 6) | (fa << 7) | (fb << 13) | (1 << 19);
        } else {
            fcode[rb] = 0;
        }
    }

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    // The CTA walks groups blockIdx.x, +G, +2G, ...; slot parities follow
    // the iteration count. Descriptors of iteration 0, synchronously:
    const int G = gridDim.x;
    if ((int)blockIdx.x < ngroups) {
        const int g0 = blockIdx.x;
        const int *src = reinterpret_cast<const int *>(a.quads + (long long)g0 * QPB);
        int *dst = reinterpret_cast<int *>(sdesc);
        constexpr int per = sizeof(QuadDesc) / 4;
        const int lim = min(QPB, a.nquad - g0 * QPB) * per;
        for (int k = tid; k < lim; k += T) dst[k] = __ldg(src + k);
    }
    __syncthreads();
    auto grp_of = [&](int it) { return (int)blockIdx.x + it * G; };
    int niter = (ngroups - (int)blockIdx.x + G - 1) / G;
    if (niter < 0) niter = 0;

    // Issue iteration `it`: its slabs (bulk copies into raw slot it&1) and
    // the next iteration's descriptors (desc slot (it+1)%3), completing on
    // bars[it&1]; then its neighbour strips (cp.async, needs its own
    // descriptors, already resident) and an L2 prefetch of its auxiliary
    // own-cell inputs.
    auto issue_iter = [&](int it) {
        int gg = grp_of(it);
        int gn = grp_of(it + 1);
        if (tid == 0) {
            uint64_t *bar = &bars[it & 1];
            int nq = (it < niter) ? min(QPB, a.nquad - gg * QPB) : 0;
            int nq1 = (it + 1 < niter) ? min(QPB, a.nquad - gn * QPB) : 0;
            unsigned bytes = (unsigned)(nq * 4 * NN * sizeof(double) * (stage_a0 ? 2 : 1) +
                                        nq1 * sizeof(QuadDesc));
            mbar_arrive_expect_tx(bar, bytes);
            double *dst = sraw + (size_t)(it & 1) * raw_slot;
            for (int ql = 0; ql < nq; ++ql)
                for (int f = 0; f < 4; ++f)
                    bulk_g2s(dst + (ql * 4 + f) * NN, a.qin + f * stride + (long long)(gg * QPB + ql) * NN,
                             (unsigned)(NN * sizeof(double)), bar);
            if (stage_a0) {
                double *dsta = saux + (size_t)(it & 1) * aux_slot;
                for (int ql = 0; ql < nq; ++ql)
                    for (int f = 0; f < 4; ++f)
                        bulk_g2s(dsta + (ql * 4 + f) * NN, a.a0 + f * stride + (long long)(gg * QPB + ql) * NN,
                                 (unsigned)(NN * sizeof(double)), bar);
            }
            if (nq1 > 0)
                bulk_g2s(sdesc + (size_t)((it + 1) % 3) * desc_slot, a.quads + (long long)gn * QPB,
                         (unsigned)(nq1 * sizeof(QuadDesc)), bar);
        }
        if (it < niter) {
            const QuadDesc *dg = sdesc + (size_t)(it % 3) * desc_slot;
            double *dst = srstrip + (size_t)(it & 1) * rstrip_slot;
            // one strip row (quad, field, side, neighbour) per SCH threads;
            // rows facing y-sides are contiguous in the neighbour's slab and
            // move as 16-byte copies, x-side rows are columns (8-byte copies)
            constexpr int SCH = (N >= 4) ? 4 : 1;     // threads per strip row
            constexpr int SPT = N / SCH;              // elements per thread
            for (int k = tid; k < QPB * 32 * SCH; k += T) {
                const int row = k / SCH;              // ((ql*4 + f)*4 + s)*2 + kk
                const int part = k - row * SCH;
                const int kk = row & 1;
                const int s = (row >> 1) & 3;
                const int f = (row >> 3) & 3;
                const int ql = row >> 5;
                if (gg * QPB + ql >= a.nquad) continue;
                const SideDesc &d = dg[ql].side[s];
                int nbr = -1;
                if (d.kind == kSideFull || d.kind == kSideFineHang) nbr = (kk == 0) ? d.nbr0 : -1;
                else if (d.kind == kSideCoarseHang) nbr = (kk == 0) ? d.nbr0 : d.nbr1;
                if (nbr < 0) continue;
                const double *src = a.qin + f * stride + (long long)nbr * NN;
                double *drow = dst + (size_t)row * N;
                const int m0 = part * SPT;
                if (s >= 2 && (SPT % 2) == 0) {
                    const int base = (s == 2) ? (N - 1) * N : 0;
#pragma unroll
                    for (int m = m0; m < m0 + SPT; m += 2) cp_async16(drow + m, src + base + m);
                } else {
#pragma unroll
                    for (int m = m0; m < m0 + SPT; ++m) cp_async8(drow + m, src + facing_cell<N>(s, m));
                }
            }
            cp_async_commit();
            if (a.a0 || a.a1) {
                constexpr int LINES = NN * 8 / 128 > 0 ? NN * 8 / 128 : 1;
                for (int k = tid; k < QPB * 4 * LINES * 2; k += T) {
                    int which = k / (QPB * 4 * LINES);
                    int r = k - which * QPB * 4 * LINES;
                    int ql = r / (4 * LINES);
                    int f = (r / LINES) % 4;
                    int ln = r % LINES;
                    const double *base = which ? a.a1 : (stage_a0 ? nullptr : a.a0);
                    if (!base || gg * QPB + ql >= a.nquad) continue;
                    prefetch_l2(base + f * stride + (long long)(gg * QPB + ql) * NN + ln * 16);
                }
            }
        }
    };

    if (niter > 0) issue_iter(0);

    for (int it = 0; it < niter; ++it) {
        const int q0 = grp_of(it) * QPB;
        // ---------------- wait for this group's data, then prefetch the next
        if (!mbar_wait_bounded(&bars[it & 1], (unsigned)((it >> 1) & 1), kWaitLimit))
            my_flags |= kFlagTimeout;
        cp_async_wait_all();
        __syncthreads();
        issue_iter(it + 1);

        const QuadDesc *sq = sdesc + (size_t)(it % 3) * desc_slot;
        const double *raw = sraw + (size_t)(it & 1) * raw_slot;
        const double *aux = saux + (size_t)(it & 1) * aux_slot;
        const double *rstrip = srstrip + (size_t)(it & 1) * rstrip_slot;

        // ---------------- phase A: per-cell records, per-quad geometry
        for (int k = tid; k < QPB * NPC; k += T) {
            int ql = k / NPC;
            int c = k - ql * NPC;
            if (q0 + ql >= a.nquad) continue;
            double q[4];
            if (c < NN) {
#pragma unroll
                for (int f = 0; f < 4; ++f) q[f] = raw[(ql * 4 + f) * NN + c];
            } else {
                int e = c - NN;   // (s*2 + kk)*N + m
                int s = e / (2 * N);
                int kk = (e / N) % 2;
                const SideDesc &d = sq[ql].side[s];
                bool present = (d.kind == kSideFull || d.kind == kSideFineHang) ? (kk == 0)
                               : (d.kind == kSideCoarseHang);
                if (!present) continue;
#pragma unroll
                for (int f = 0; f < 4; ++f) q[f] = rstrip[ql * 4 * S::NSTRIP + f * S::NSTRIP + e];
            }
            alignas(16) R P[RS];
            FluxOps::prims(q, P);
            typename Tr::V *dst = reinterpret_cast<typename Tr::V *>(prim + (size_t)(ql * NPC + c) * RS);
#pragma unroll
            for (int v = 0; v < Tr::nv; ++v) dst[v] = reinterpret_cast<const typename Tr::V *>(P)[v];
        }
        // per quad: rectangle spacing (FP32 form: x-face normal (hy,0),
        // y-face normal (0,hx), volume hx*hy) and each side's cell_h
        if (tid < 4 * QPB) {
            const int ql = tid >> 2, s = tid & 3;
            if (q0 + ql < a.nquad) {
                geo[8 * ql + 4 + s] = cell_h_of(a.h_base, sq[ql].side[s].level, N);
                if (F32 && s == 0) {
                    const double *g = sq[ql].corner;
                    double hx = (g[2] - g[0]) / (double)N, hy = (g[5] - g[1]) / (double)N;
                    geo[8 * ql + 0] = hx;
                    geo[8 * ql + 1] = hy;
                    geo[8 * ql + 2] = 1.0 / (hx * hy);
                    geo[8 * ql + 3] = hx * hy;
                }
            }
        }
        if (!F32) {
            // The FP64 form takes normals and volumes from the (n+1)^2
            // bilinear nodes, exactly as the reference.
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
        }
        __syncthreads();

        // ---------------- phase B: face fluxes
        // Faces of a quad: x-faces (row fb, position fa = 0..N) then y-faces
        // (position fa = 0..N, column fb); fa = 0 / N are the edge faces.
        // Edge and interior faces only differ in where the two states and
        // the normal come from, so a warp mixing them runs one flux code
        // path (only physical-boundary faces take the bc branch).
#pragma unroll
        for (int rb = 0; rb < RB; ++rb) {
            const int code = fcode[rb];
            if (!(code >> 19)) continue;
            const int ql = code & 63;
            if (q0 + ql >= a.nquad) continue;
            const bool xd = (code >> 6) & 1;
            const int fa = (code >> 7) & 63;
            const int fb = (code >> 13) & 63;
            const R *pq = prim + (size_t)ql * NPC * RS;
            int li, ri, bcv = -1;
            R n0, n1;
            if (fa == 0 || fa == N) {
                const int s = (xd ? 0 : 2) + (fa == N ? 1 : 0);
                const SideDesc &d = sq[ql].side[s];
                const int own = xd ? (fb * N + (fa == 0 ? 0 : N - 1)) : ((fa == 0 ? 0 : N - 1) * N + fb);
                const int nb = NN + (s * 2) * N + fb;
                const R h = (R)geo[8 * ql + 4 + s];
                if (d.kind == kSideBoundary) {
                    bcv = d.bc;
                    li = own;
                    ri = own;
                    n0 = xd ? (fa == 0 ? -h : h) : (R)0;
                    n1 = xd ? (R)0 : (fa == 0 ? -h : h);
                } else {
                    li = (s & 1) ? own : nb;
                    ri = (s & 1) ? nb : own;
                    n0 = xd ? h : (R)0;
                    n1 = xd ? (R)0 : h;
                }
            } else {
                li = xd ? (fb * N + fa - 1) : ((fa - 1) * N + fb);
                ri = xd ? (fb * N + fa) : (fa * N + fb);
                if (F32) {
                    n0 = xd ? (R)geo[8 * ql + 1] : (R)0;
                    n1 = xd ? (R)0 : (R)geo[8 * ql + 0];
                } else {
                    const double *nd = nodes + ql * NP1 * NP1 * 2;
                    const double *p1 = xd ? nd + 2 * (fb * NP1 + fa) : nd + 2 * (fa * NP1 + fb + 1);
                    const double *p2 = xd ? nd + 2 * ((fb + 1) * NP1 + fa) : nd + 2 * (fa * NP1 + fb);
                    n0 = (R)(p2[1] - p1[1]);
                    n1 = (R)(p1[0] - p2[0]);
                }
            }
            alignas(16) R Lp[RS];
            alignas(16) R Rp[RS];
            alignas(16) R fl[4];
            load_rec<F32>(pq, li, Lp);
            load_rec<F32>(pq, ri, Rp);
            if (bcv < 0) {
                if (xd) FluxOps::template roe_axis<0>(Lp, Rp, n0, n1, fl);
                else FluxOps::template roe_axis<1>(Lp, Rp, n0, n1, fl);
            } else {
                R qin[4] = {(R)a.qinflow[0], (R)a.qinflow[1], (R)a.qinflow[2], (R)a.qinflow[3]};
                FluxOps::bc(bcv, Lp, n0, n1, qin, fl);
                // FP32 form: a low-side boundary face is stored with the
                // sign of the interior faces' convention (flux towards +x /
                // +y), so that every cell sums its four faces alike
                if (F32 && fa == 0) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) fl[f] = -fl[f];
                }
            }
            if (xd) store_flux<F32>(fx, (ql * N + fb) * NP1 + fa, fl);
            else store_flux<F32>(fy, (ql * NP1 + fa) * N + fb, fl);
        }
        // second flux of each coarse hanging edge cell (only at level jumps)
        bool any_hang = false;
#pragma unroll
        for (int ql = 0; ql < QPB; ++ql)
#pragma unroll
            for (int s = 0; s < 4; ++s)
                any_hang |= (q0 + ql < a.nquad) && sq[ql].side[s].kind == kSideCoarseHang;
        if (any_hang) {
            for (int k = tid; k < QPB * 4 * N; k += T) {
                const int ql = k / (4 * N);
                const int s = (k / N) % 4;
                const int m = k % N;
                if (q0 + ql >= a.nquad) continue;
                const SideDesc &d = sq[ql].side[s];
                if (d.kind != kSideCoarseHang) continue;
                const R *pq = prim + (size_t)ql * NPC * RS;
                const bool xd = s < 2;
                const int own = xd ? (m * N + (s == 0 ? 0 : N - 1)) : ((s == 2 ? 0 : N - 1) * N + m);
                const int nb = NN + (s * 2 + 1) * N + m;
                const R h = (R)geo[8 * ql + 4 + s];
                alignas(16) R Lp[RS];
                alignas(16) R Rp[RS];
                alignas(16) R fl[4];
                load_rec<F32>(pq, (s & 1) ? own : nb, Lp);
                load_rec<F32>(pq, (s & 1) ? nb : own, Rp);
                if (xd) FluxOps::template roe_axis<0>(Lp, Rp, h, (R)0, fl);
                else FluxOps::template roe_axis<1>(Lp, Rp, (R)0, h, fl);
                store_flux<F32>(fh, (ql * 4 + s) * N + m, fl);
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
            double F[4];
            if constexpr (F32) {
                // FP32-flux form: -F(x-1/2) +F(x+1/2) -F(y-1/2) +F(y+1/2),
                // edge faces included (low-side boundary faces were stored
                // negated), summed in FP64; a coarse hanging edge adds its
                // second flux with the edge's sign.
                double G[4];
                load_flux<F32>(fx, (ql * N + j) * NP1 + i, F);
                load_flux<F32>(fx, (ql * N + j) * NP1 + i + 1, G);
#pragma unroll
                for (int f = 0; f < 4; ++f) r[f] = G[f] - F[f];
                load_flux<F32>(fy, (ql * NP1 + j) * N + i, F);
                load_flux<F32>(fy, (ql * NP1 + j + 1) * N + i, G);
#pragma unroll
                for (int f = 0; f < 4; ++f) r[f] = (r[f] - F[f]) + G[f];
                if (any_hang) {
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const bool on = (s == 0) ? i == 0 : (s == 1) ? i == N - 1 : (s == 2) ? j == 0 : j == N - 1;
                        if (!on || qd.side[s].kind != kSideCoarseHang) continue;
                        load_flux<F32>(fh, (ql * 4 + s) * N + ((s < 2) ? j : i), F);
#pragma unroll
                        for (int f = 0; f < 4; ++f) r[f] = (s & 1) ? r[f] + F[f] : r[f] - F[f];
                    }
                }
            } else {
                int sx = (i == 0) ? 0 : (i == N - 1) ? 1 : -1;
                int sy = (j == 0) ? 2 : (j == N - 1) ? 3 : -1;
                int first = sx, second = sy;
                if (sx >= 0 && sy >= 0 && qd.side[sy].rank < qd.side[sx].rank) { first = sy; second = sx; }
#pragma unroll
                for (int pass = 0; pass < 2; ++pass) {
                    int s = pass == 0 ? first : second;
                    if (s < 0) continue;
                    int kind = qd.side[s].kind;
                    int m = (s < 2) ? j : i;
                    if (s < 2) load_flux<F32>(fx, (ql * N + j) * NP1 + (s == 0 ? 0 : N), F);
                    else load_flux<F32>(fy, (ql * NP1 + (s == 2 ? 0 : N)) * N + i, F);
                    double F2[4] = {0.0, 0.0, 0.0, 0.0};
                    if (kind == kSideCoarseHang) load_flux<F32>(fh, (ql * 4 + s) * N + m, F2);
                    if (kind == kSideBoundary || (s & 1)) {
#pragma unroll
                        for (int f = 0; f < 4; ++f) {
                            r[f] = r[f] + F[f];
                            if (kind == kSideCoarseHang) r[f] = r[f] + F2[f];
                        }
                    } else {
#pragma unroll
                        for (int f = 0; f < 4; ++f) {
                            r[f] = r[f] - F[f];
                            if (kind == kSideCoarseHang) r[f] = r[f] - F2[f];
                        }
                    }
                }
                if (i > 0) {
                    load_flux<F32>(fx, (ql * N + j) * NP1 + i, F);
#pragma unroll
                    for (int f = 0; f < 4; ++f) r[f] = r[f] - F[f];
                }
                if (i < N - 1) {
                    load_flux<F32>(fx, (ql * N + j) * NP1 + i + 1, F);
#pragma unroll
                    for (int f = 0; f < 4; ++f) r[f] = r[f] + F[f];
                }
                if (j > 0) {
                    load_flux<F32>(fy, (ql * NP1 + j) * N + i, F);
#pragma unroll
                    for (int f = 0; f < 4; ++f) r[f] = r[f] - F[f];
                }
                if (j < N - 1) {
                    load_flux<F32>(fy, (ql * NP1 + j + 1) * N + i, F);
#pragma unroll
                    for (int f = 0; f < 4; ++f) r[f] = r[f] + F[f];
                }
            }
            double vol;
            double kv[4];
            if (F32) {
                vol = geo[8 * ql + 3];
                const double inv = geo[8 * ql + 2];
#pragma unroll
                for (int f = 0; f < 4; ++f) kv[f] = -(r[f] * inv);
            } else {
                const double *nd = nodes + ql * NP1 * NP1 * 2;
                const double *n1p = nd + 2 * (j * NP1 + i);
                const double *n3p = nd + 2 * ((j + 1) * NP1 + i);
                vol = subcell_volume(n1p[0], n1p[1], n1p[2], n1p[3], n3p[0], n3p[1], n3p[2], n3p[3]);
#pragma unroll
                for (int f = 0; f < 4; ++f) kv[f] = (r[f] / vol) * -1.0;
            }

            const long long gi = (long long)(q0 + ql) * NN + c;
            // the first auxiliary input: staged in shared memory (FP32 form)
            // or read from HBM
            auto A0 = [&](int f) -> double {
                if constexpr (F32) return aux[(ql * 4 + f) * NN + c];
                else return a.a0[f * stride + gi];
            };
            double q0v[4], qn[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) q0v[f] = raw[(ql * 4 + f) * NN + c];

            auto A1 = [&](int f) -> double { return a.a1[f * stride + gi]; };
            rk_update(a, dt, stride, gi, q0v, kv, A0, A1, qn);

            if (a.last_stage) {
#pragma unroll
                for (int f = 0; f < 4; ++f) my_norm += kv[f] * kv[f];
                if (a.cfl_on) {
                    double cand = FluxOps::cfl(qn, vol, a.cfl);
                    if (cand < my_dt_min) my_dt_min = cand;
                }
                double rho = qn[0];
                double pe = qn[3] * rho - 0.5 * (qn[1] * qn[1] + qn[2] * qn[2]);
                if (!(rho > 0.0) || !(pe > 0.0)) my_flags |= kFlagNegative;
            }
        }
        __syncthreads();
    }

    // ---------------- block reductions: CFL min (one atomic per block), the
    // residual norm (per-block partials, summed by the last block to finish
    // in a fixed order -- strided per thread, then warp and block trees -- so
    // the result does not depend on scheduling), flags.
    __shared__ int s_last;
    const int lane = tid & 31, warp = tid >> 5;
    int wflags = __reduce_or_sync(0xffffffffu, my_flags);
    if (wflags && lane == 0) atomicOr(&a.scal->flags, wflags);
    if (!a.last_stage) return;
    double wmin = warp_min(my_dt_min);
    double wsum = warp_sum(my_norm);
    if (lane == 0) { red[warp] = wmin; red[32 + warp] = wsum; }
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
        const unsigned ticket = atomicAdd(&a.scal->done_blocks, 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double part = 0.0;
    for (int b = tid; b < (int)gridDim.x; b += T) part += __ldcg(a.partials + b);
    part = warp_sum(part);
    if (lane == 0) red[warp] = part;
    __syncthreads();
    if (tid == 0) {
        double tot = red[0];
        for (int w = 1; w < T / 32; ++w) tot += red[w];
        a.scal->norm_sq = tot;
        if (!isfinite(tot)) atomicOr(&a.scal->flags, kFlagNonFinite);
        a.scal->done_blocks = 0u;
    }
}

}  // namespace amrgpu
