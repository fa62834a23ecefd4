// stage_sweep64.cuh -- the plain FP64 form's RK stage for 16x16 and 8x8
// patches as a row sweep: one warp per 16x16 quadrant (two per warp for
// 8x8), no block-wide barriers.
//
// It produces the same bits as stage_kernel<n, ..., FP64> and therefore as
// the reference: the same flux code (flux_roe_2d, flux_2d_module.F90:63-182,
// on records made by the flux's own expressions; boundary flux
// bc_2d_module.F90:14-75), interior face normals and sub-cell volumes from
// the same bilinear nodes (bilinear_node_2d_module.F90:14-36,
// solver_residual_subgrid_2d_module.F90:82-163), edge normals from cell_h
// of the side's level, and each cell's residual summed in the reference's
// order (physics_rhs_structured.c:73-276: the edge faces first, in face_info
// order, a coarse hanging edge's two fluxes one after the other; then
// solver_residual_subgrid_2d's interior faces -F(x-1/2) +F(x+1/2) -F(y-1/2)
// +F(y+1/2)), divided by the volume and negated, then the stage update with
// the reference's coefficients (rk_time_integrators.c). This translation
// unit is compiled with -fmad=false, so no multiply-add is contracted.
//
//   lane = (sub, h, i): quad sub of the warp's 32/(2N) quads, column i,
//        rows R*h .. R*h+R-1 with R = N/2.
//   edges   each lane evaluates one edge face per round (sides 0/1, then
//           2/3; a coarse hanging edge also its second, index-paired flux)
//           into a per-warp table, and the faces between rows R-1 and R;
//   sweep   at step t lane (i, h) takes cell (i, j = Rh+t): its record, the
//           bilinear nodes of row j+1 at columns i and i+1 (row j's came
//           from the step before), then two flux evaluations through one
//           call site -- the x-face at i-1/2 with the left neighbour's record
//           taken by a warp shuffle (its value goes to lane i-1, which needs
//           it as its i+1/2 face, by a second shuffle), then the y-face at
//           j-1/2 with the record of row j-1, which completes row j-1 (its
//           update is written).
//
// Registers are the limit of an FP64 flux kernel (a flux evaluation holds
// about 60 live doubles), so what a lane carries from one row to the next --
// row j-1's record, partial residual, input state and volume -- waits in
// shared memory, and the row's own-cell inputs (the next row's state, the
// stage's auxiliary inputs) arrive there by cp.async one step ahead of use.
#pragma once

#include "async_copy.cuh"
#include "flux_fp64.cuh"
#include "stage_kernel.cuh"
#include "sweep_common.cuh"

namespace amrgpu {

// Dynamic shared memory of the FP64 sweep, in doubles per warp.
template <int N>
struct Sweep64Smem {
    static constexpr int QPW = 32 / (2 * N);
    static constexpr int RS = 9;                      // record: rho, rho u, rho v, rho E, u, v, p, H, sqrt(rho)
    static constexpr int edge = QPW * 4 * 2 * N * 4;  // [quad][side][first/second flux][position][field]
    static constexpr int mid = QPW * N * 4;           // [quad][column][field]: faces between rows R-1 and R
    static constexpr int carry = (RS + 4 + 4 + 1) * 32;  // [record, partial, input state, volume][lane]
    static constexpr int qbuf = 4 * 32;                  // next row's state [field][lane]
    static constexpr int abuf = 8 * 32;                  // auxiliary inputs a0, a1 [field][lane]
    static constexpr int o_edge = 0, o_mid = o_edge + edge, o_carry = o_mid + mid, o_q = o_carry + carry,
                         o_a = o_q + qbuf;
    static constexpr int per_warp = o_a + abuf;
    static constexpr size_t bytes(int warps) { return sizeof(double) * (size_t)per_warp * (size_t)warps; }
};

// ST = 0: any scheme and stage, read from the arguments; ST = 1..3: stage
// ST of the reference's RK3 (the FP64 form's default scheme) fixed at
// compile time -- the same update expressions without the per-cell switch.
template <int N, int WARPS, int ST>
__device__ __forceinline__ void sweep64_body(const StageArgs &a)
{
    static_assert(N == 16 || N == 8, "row sweep for 16x16 and 8x8 patches");
    using S = Sweep64Smem<N>;
    constexpr int NN = N * N;
    constexpr int QPW = S::QPW;
    constexpr int R = N / 2;  // rows per half-patch
    constexpr int RS = S::RS;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) double sm64[];
    __shared__ double red[64];
    __shared__ int s_last;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int sub = lane / (2 * N), l = lane % (2 * N);
    const int i = l % N, h = l / N;
    const long long stride = a.stride;
    const double scale_factor = 2.0 / (double)N;
    const double xi0 = scale_factor * (double)i - 1.0;        // nodes at column i
    const double xi1 = scale_factor * (double)(i + 1) - 1.0;  // ... and i+1

    double *wsm = sm64 + (size_t)w * S::per_warp;
    double(*sedge)[4][2][N][4] = reinterpret_cast<double(*)[4][2][N][4]>(wsm + S::o_edge);
    double(*smid)[N][4] = reinterpret_cast<double(*)[N][4]>(wsm + S::o_mid);
    double *car = wsm + S::o_carry + lane;  // slot c at car[32 c]
    double *qb = wsm + S::o_q + lane;       // field f at qb[32 f]
    double *ab = wsm + S::o_a + lane;       // a0 field f at ab[32 f], a1 at ab[32 (4 + f)]
    enum { kPart = RS, kQ = RS + 4, kVol = RS + 8 };

    const double dt = sweep_step_dt(a);
    double my_dt_min = a.dt_cap;
    double my_norm = 0.0;
    int my_flags = 0;
    // the reference RK3's auxiliary inputs: none in stage 1, Q0 and k1 in
    // stage 2, the combination C in stage 3
    const bool has_a0 = ST > 0 ? ST >= 2 : a.a0 != nullptr;
    const bool has_a1 = ST > 0 ? ST == 2 : a.a1 != nullptr;

    // work items as in the FP32 sweep: first by warp index, then from the
    // quad counter; a quad past the end is computed on the item's first
    // quad and neither stored nor reduced
    const int nwarps = gridDim.x * WARPS;
    const int nitems = (a.nquad + QPW - 1) / QPW;
    int item = blockIdx.x * WARPS + w;
    while (item < nitems) {
        const bool valid = QPW == 1 || item * QPW + sub < a.nquad;
        const int quad = valid ? item * QPW + sub : item * QPW;
        const QuadDesc &qd = a.quads[quad];
        const double *g = qd.corner;
        const double *Qq = a.qin + (long long)quad * NN;
        auto load_rec = [&](const double *base, int cell, double P[RS]) {
            double q[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) q[f] = base[f * stride + cell];
            cell_prims_fp64(q, P);
        };
        // the first row's state, on its way while the edges are computed
#pragma unroll
        for (int f = 0; f < 4; ++f) cp_async8(qb + 32 * f, Qq + f * stride + (R * h) * N + i);
        cp_async_commit();
        cp_async_commit();  // (no auxiliary group before the first row)

        // ---------------- edges: round 0 sides 0 / 1, round 1 sides 2 / 3
#pragma unroll 1
        for (int round = 0; round < 2; ++round) {
            const int s = 2 * round + h, m = i;
            const bool xd = round == 0;
            const SideDesc d = qd.side[s];
            const int own = (s == 0) ? m * N : (s == 1) ? m * N + N - 1 : (s == 2) ? m : (N - 1) * N + m;
            double Po[RS], fl[4];
            load_rec(Qq, own, Po);
            const double hc = cell_h_of(a.h_base, d.level, N);
            if (d.kind == kSideBoundary) {
                const double n0 = xd ? ((s & 1) ? hc : -hc) : 0.0;
                const double n1 = xd ? 0.0 : ((s & 1) ? hc : -hc);
                bc_flux_fp64(d.bc, Po, n0, n1, a.qinflow, fl);
#pragma unroll
                for (int f = 0; f < 4; ++f) sedge[sub][s][0][m][f] = fl[f];
            } else {
                // the neighbour's facing cell at the same position (a coarse
                // hanging edge pairs it with both fine quads)
                const int fc = facing_cell<N>(s, m);
                const int nk = (d.kind == kSideCoarseHang) ? 2 : 1;
                const double n0 = xd ? hc : 0.0, n1 = xd ? 0.0 : hc;
#pragma unroll 1
                for (int k = 0; k < nk; ++k) {
                    double Pn[RS], Lr[RS], Rr[RS];
                    load_rec(a.qin + (long long)(k == 0 ? d.nbr0 : d.nbr1) * NN, fc, Pn);
#pragma unroll
                    for (int c = 0; c < RS; ++c) {
                        Lr[c] = (s & 1) ? Po[c] : Pn[c];
                        Rr[c] = (s & 1) ? Pn[c] : Po[c];
                    }
                    roe_flux_prim_fp64(Lr, Rr, n0, n1, fl);
#pragma unroll
                    for (int f = 0; f < 4; ++f) sedge[sub][s][k][m][f] = fl[f];
                }
            }
        }
        // ---------------- the faces between rows R-1 and R (column i):
        // normal from the nodes (i+1, R) and (i, R)
        {
            double P[RS], O[RS], fl[4];
            load_rec(Qq, (R - 1 + h) * N + i, P);
#pragma unroll
            for (int c = 0; c < RS; ++c) O[c] = __shfl_xor_sync(FULL, P[c], N);
            if (h == 0) {
                const double eta = scale_factor * (double)R - 1.0;
                double x1, y1, x2, y2;
                bilinear_node(g, xi1, eta, x1, y1);
                bilinear_node(g, xi0, eta, x2, y2);
                roe_flux_prim_fp64(P, O, y2 - y1, x1 - x2, fl);
#pragma unroll
                for (int f = 0; f < 4; ++f) smid[sub][i][f] = fl[f];
            }
        }
        __syncwarp();

        // the edge contributions of cell (i, j) in face_info order, starting
        // from 0 (physics_rhs_structured.c:73-262 visits faces in order)
        auto edge_sum = [&](int j, double r[4]) {
            const int sx = (i == 0) ? 0 : (i == N - 1) ? 1 : -1;
            const int sy = (j == 0) ? 2 : (j == N - 1) ? 3 : -1;
            if (sx < 0 && sy < 0) return;
            int first = sx, second = sy;
            if (sx >= 0 && sy >= 0 && qd.side[sy].rank < qd.side[sx].rank) {
                first = sy;
                second = sx;
            }
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                const int s = pass == 0 ? first : second;
                if (s < 0) continue;
                const int kind = qd.side[s].kind;
                const int m = (s < 2) ? j : i;
                const bool hang = kind == kSideCoarseHang;
                const double *F = sedge[sub][s][0][m];
                const double *F2 = sedge[sub][s][1][m];
                if (kind == kSideBoundary || (s & 1)) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        r[f] = r[f] + F[f];
                        if (hang) r[f] = r[f] + F2[f];
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        r[f] = r[f] - F[f];
                        if (hang) r[f] = r[f] - F2[f];
                    }
                }
            }
        };
        // finishes row jr from the carried state: + F(y+1/2) when that face
        // is interior, / volume, x -1, stage update with the auxiliary
        // inputs in ab, last-stage reductions
        auto finish = [&](int jr, const double *gup) {
            const long long gi = (long long)quad * NN + jr * N + i;
            const double vol = car[32 * kVol];
            double kv[4], qn[4], q0v[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const double p = car[32 * (kPart + f)];
                const double r = gup ? p + gup[f] : p;
                kv[f] = (r / vol) * -1.0;
                q0v[f] = car[32 * (kQ + f)];
            }
            if (!valid) return;
            auto A0 = [&](int f) -> double { return ab[32 * f]; };
            auto A1 = [&](int f) -> double { return ab[32 * (4 + f)]; };
            if constexpr (ST > 0) rk_update<kSchemeRK3, ST>(a, dt, stride, gi, q0v, kv, A0, A1, qn);
            else rk_update(a, dt, stride, gi, q0v, kv, A0, A1, qn);
            if (ST > 0 ? ST == 3 : a.last_stage != 0) {
#pragma unroll
                for (int f = 0; f < 4; ++f) my_norm += kv[f] * kv[f];
                if (a.cfl_on) {
                    const double cand = cfl_candidate_fp64(qn, vol, a.cfl);
                    if (cand < my_dt_min) my_dt_min = cand;
                }
                const double rho = qn[0];
                const double pe = qn[3] * rho - 0.5 * (qn[1] * qn[1] + qn[2] * qn[2]);
                if (!(rho > 0.0) || !(pe > 0.0)) my_flags |= kFlagNegative;
            }
        };
        // the auxiliary inputs of row jr into ab (one cp.async group)
        auto fetch_aux = [&](int jr) {
            const long long gi = (long long)quad * NN + jr * N + i;
            if (has_a0) {
#pragma unroll
                for (int f = 0; f < 4; ++f) cp_async8(ab + 32 * f, a.a0 + f * stride + gi);
            }
            if (has_a1) {
#pragma unroll
                for (int f = 0; f < 4; ++f) cp_async8(ab + 32 * (4 + f), a.a1 + f * stride + gi);
            }
            cp_async_commit();
        };

        // ---------------- sweep over the lane's R rows. cp.async groups in
        // flight at the start of step t: the state of row j (issued one step
        // earlier) and the auxiliary inputs of row j-1.
        double xa, ya, xb, yb;  // nodes (i, j) and (i+1, j) of the current row
        {
            const double eta = scale_factor * (double)(R * h) - 1.0;
            bilinear_node(g, xi0, eta, xa, ya);
            bilinear_node(g, xi1, eta, xb, yb);
        }
#pragma unroll 1
        for (int t = 0; t < R; ++t) {
            const int j = R * h + t;
            cp_async_wait_group<1>();  // row j's state has landed
            double q4[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) q4[f] = qb[32 * f];
            double P[RS];
            cell_prims_fp64(q4, P);
            // the next row's state into the buffer just read (the record
            // above consumed it)
            if (t < R - 1) {
#pragma unroll
                for (int f = 0; f < 4; ++f) cp_async8(qb + 32 * f, Qq + f * stride + (j + 1) * N + i);
            }
            cp_async_commit();
            // nodes (i, j+1), (i+1, j+1), the cell's volume and x-face normal
            double xc, yc, xd, yd;
            {
                const double eta = scale_factor * (double)(j + 1) - 1.0;
                bilinear_node(g, xi0, eta, xc, yc);
                bilinear_node(g, xi1, eta, xd, yd);
            }
            const double vol = subcell_volume(xa, ya, xb, yb, xc, yc, xd, yd);
            double r[4];
            // k = 0: x-face at i-1/2, nodes (i, j) -> (i, j+1), the left
            //        neighbour's record (lane i = 0's is an edge face);
            // k = 1: y-face at j-1/2, nodes (i+1, j) -> (i, j), row j-1's
            //        record, which completes row j-1
            const int nk = (t > 0) ? 2 : 1;
#pragma unroll 1
            for (int k = 0; k < nk; ++k) {
                double A[RS];
                double n0, n1;
                if (k == 0) {
#pragma unroll
                    for (int c = 0; c < RS; ++c) A[c] = __shfl_up_sync(FULL, P[c], 1, N);
                    n0 = yc - ya;
                    n1 = xa - xc;
                } else {
#pragma unroll
                    for (int c = 0; c < RS; ++c) A[c] = car[32 * c];
                    n0 = ya - yb;
                    n1 = xb - xa;
                }
                double F[4];
                roe_flux_prim_fp64(A, P, n0, n1, F);
                if (k == 0) {
                    double Fr[4];
#pragma unroll
                    for (int f = 0; f < 4; ++f) Fr[f] = __shfl_down_sync(FULL, F[f], 1, N);
#pragma unroll
                    for (int f = 0; f < 4; ++f) r[f] = 0.0;
                    edge_sum(j, r);
                    // interior x-faces only (lane 0's low and lane N-1's high
                    // face are edge faces, summed above): each sum is
                    // formed and kept or dropped by a select, not a branch
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        const double rl = r[f] - F[f];
                        r[f] = i > 0 ? rl : r[f];
                        const double rr = r[f] + Fr[f];
                        r[f] = i < N - 1 ? rr : r[f];
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 4; ++f) r[f] = r[f] - F[f];
                    cp_async_wait_group<1>();  // row j-1's auxiliary inputs
                    finish(j - 1, F);
                }
            }
            if (t == 0 && h == 1) {
#pragma unroll
                for (int f = 0; f < 4; ++f) r[f] = r[f] - smid[sub][i][f];
            }
            fetch_aux(j);
            // carry row j to the next step
#pragma unroll
            for (int c = 0; c < RS; ++c) car[32 * c] = P[c];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                car[32 * (kPart + f)] = r[f];
                car[32 * (kQ + f)] = q4[f];
            }
            car[32 * kVol] = vol;
            xa = xc;
            ya = yc;
            xb = xd;
            yb = yd;
        }
        // the half's top row: the face between rows R-1 and R (h = 0) or the
        // patch's top edge, already summed (h = 1)
        cp_async_wait_group<0>();
        finish(R * h + R - 1, h == 0 ? smid[sub][i] : nullptr);
        __syncwarp();  // the next item rewrites this warp's tables
        unsigned nxt = 0;
        if (lane == 0) nxt = atomicAdd(&a.scal->work_next, 1u);
        item = nwarps + (int)__shfl_sync(FULL, nxt, 0);
    }

    sweep_reduce<WARPS>(a, my_dt_min, my_norm, my_flags, red, &s_last);
}

template <int WARPS, int MINB, int ST = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB) sweep64_16_kernel(const StageArgs a)
{
    stage_launch_gate();
    sweep64_body<16, WARPS, ST>(a);
}

template <int WARPS, int MINB, int ST = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB) sweep64_8_kernel(const StageArgs a)
{
    stage_launch_gate();
    sweep64_body<8, WARPS, ST>(a);
}

}  // namespace amrgpu
