// stage_sweep64.cuh -- the plain FP64 form's RK stage for 16x16 and 8x8
// patches as a row sweep: one warp per 16x16 quadrant (two per warp for
// 8x8), per-cell records in registers, no block-wide barriers.
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
//   sweep   at step t lane (i, h) loads cell (i, j = Rh+t) and builds its
//           record; it first completes row j-1 (the y-face flux at j-1/2
//           with the record it kept of row j-1, then that row's update),
//           then computes the bilinear nodes of row j+1 at columns i and i+1
//           (row j's came from the step before), the x-face flux at i-1/2
//           with the left neighbour's record taken by a warp shuffle, and
//           hands it to lane i-1 (its i+1/2 face) by a second shuffle. The
//           two flux evaluations of a step thus never hold their operands at
//           the same time (168 registers, 12 warps per SM).
#pragma once

#include "flux_fp64.cuh"
#include "stage_kernel.cuh"
#include "sweep_common.cuh"

namespace amrgpu {

template <int N, int WARPS>
__device__ __forceinline__ void sweep64_body(const StageArgs &a)
{
    static_assert(N == 16 || N == 8, "row sweep for 16x16 and 8x8 patches");
    constexpr int NN = N * N;
    constexpr int QPW = 32 / (2 * N);  // quads per warp
    constexpr int R = N / 2;           // rows per half-patch
    constexpr int RS = 9;              // record: rho, rho u, rho v, rho E, u, v, p, H, sqrt(rho)
    constexpr unsigned FULL = 0xffffffffu;
    // per warp and quad: edge fluxes [side][first / second (coarse hanging
    // edge) flux][position][field] and the faces between rows R-1 and R
    __shared__ double sedge[WARPS][QPW][4][2][N][4];
    __shared__ double smid[WARPS][QPW][N][4];
    __shared__ double red[64];
    __shared__ int s_last;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int sub = lane / (2 * N), l = lane % (2 * N);
    const int i = l % N, h = l / N;
    const long long stride = a.stride;
    const double scale_factor = 2.0 / (double)N;
    const double xi0 = scale_factor * (double)i - 1.0;        // nodes at column i
    const double xi1 = scale_factor * (double)(i + 1) - 1.0;  // ... and i+1

    const double dt = sweep_step_dt(a);
    double my_dt_min = a.dt_cap;
    double my_norm = 0.0;
    int my_flags = 0;

    // work items as in the FP32 sweep: first by warp index, then from the
    // quad counter; a quad past the end is computed on the item's first
    // quad and neither stored nor reduced
    const int nwarps = gridDim.x * WARPS;
    const int nitems = (a.nquad + QPW - 1) / QPW;
    int item = blockIdx.x * WARPS + w;
    while (item < nitems) {
        const bool valid = item * QPW + sub < a.nquad;
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

        // ---------------- edges: round 0 sides 0 / 1, round 1 sides 2 / 3
#pragma unroll
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
                for (int f = 0; f < 4; ++f) sedge[w][sub][s][0][m][f] = fl[f];
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
                    for (int f = 0; f < 4; ++f) sedge[w][sub][s][k][m][f] = fl[f];
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
                for (int f = 0; f < 4; ++f) smid[w][sub][i][f] = fl[f];
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
            if (sx >= 0 && sy >= 0 && qd.side[sy].rank < qd.side[sx].rank) { first = sy; second = sx; }
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                const int s = pass == 0 ? first : second;
                if (s < 0) continue;
                const int kind = qd.side[s].kind;
                const int m = (s < 2) ? j : i;
                const bool hang = kind == kSideCoarseHang;
                const double *F = sedge[w][sub][s][0][m];
                const double *F2 = sedge[w][sub][s][1][m];
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

        // ---------------- sweep over the lane's R rows
        // A step first completes the row below (its y-face flux, then the
        // update) and only then evaluates its own x-face flux, so that the
        // two flux evaluations never hold their operands at the same time.
        double below[RS];  // record of the row below (partner of the y-face)
        double part[4];    // residual of the row below without its face at j+1/2
        double qbelow[4];  // input state of the row below
        double volbelow = 0.0;
        const bool has_a0 = a.a0 != nullptr;
        // finishes row jr: + F(y+1/2) when that face is interior, / volume,
        // x -1, stage update, last-stage reductions; a0 is the row's first
        // auxiliary input
        auto finish = [&](int jr, const double *gup, const double a0r[4]) {
            const long long gi = (long long)quad * NN + jr * N + i;
            double kv[4], qn[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const double r = gup ? part[f] + gup[f] : part[f];
                kv[f] = (r / volbelow) * -1.0;
            }
            if (!valid) return;
            auto A0 = [&](int f) -> double { return a0r[f]; };
            rk_update(a, dt, stride, gi, qbelow, kv, A0, qn);
            if (a.last_stage) {
#pragma unroll
                for (int f = 0; f < 4; ++f) my_norm += kv[f] * kv[f];
                if (a.cfl_on) {
                    const double cand = cfl_candidate_fp64(qn, volbelow, a.cfl);
                    if (cand < my_dt_min) my_dt_min = cand;
                }
                const double rho = qn[0];
                const double pe = qn[3] * rho - 0.5 * (qn[1] * qn[1] + qn[2] * qn[2]);
                if (!(rho > 0.0) || !(pe > 0.0)) my_flags |= kFlagNegative;
            }
        };
        auto load_a0 = [&](int jr, double a0r[4]) {
#pragma unroll
            for (int f = 0; f < 4; ++f)
                a0r[f] = has_a0 ? a.a0[f * stride + (long long)quad * NN + jr * N + i] : 0.0;
        };
        // nodes (i, j) and (i+1, j) of the current row
        double xa, ya, xb, yb;
        {
            const double eta = scale_factor * (double)(R * h) - 1.0;
            bilinear_node(g, xi0, eta, xa, ya);
            bilinear_node(g, xi1, eta, xb, yb);
        }
        double qnext[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) qnext[f] = Qq[f * stride + (R * h) * N + i];
#pragma unroll 1
        for (int t = 0; t < R; ++t) {
            const int j = R * h + t;
            double q4[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) q4[f] = qnext[f];
            if (t < R - 1) {
#pragma unroll
                for (int f = 0; f < 4; ++f) qnext[f] = Qq[f * stride + (j + 1) * N + i];
            }
            double P[RS];
            cell_prims_fp64(q4, P);
            // y-face at j-1/2: nodes (i+1, j) -> (i, j); completes row j-1
            double fy[4];
            const bool has_fy = j > 0;
            if (t == 0) {
                if (h == 1) {
#pragma unroll
                    for (int f = 0; f < 4; ++f) fy[f] = smid[w][sub][i][f];
                }
            } else {
                double a0r[4];
                load_a0(j - 1, a0r);
                roe_flux_prim_fp64(below, P, ya - yb, xb - xa, fy);
                finish(j - 1, fy, a0r);
            }
            // nodes (i, j+1), (i+1, j+1) and the cell's volume
            double xc, yc, xd, yd;
            {
                const double eta = scale_factor * (double)(j + 1) - 1.0;
                bilinear_node(g, xi0, eta, xc, yc);
                bilinear_node(g, xi1, eta, xd, yd);
            }
            const double n0x = yc - ya, n1x = xa - xc;
            volbelow = subcell_volume(xa, ya, xb, yb, xc, yc, xd, yd);
            xa = xc; ya = yc; xb = xd; yb = yd;
            // x-face at i-1/2: nodes (i, j) -> (i, j+1); lane i = 0's is an edge face
            double L[RS], fx[4], fxr[4];
#pragma unroll
            for (int c = 0; c < RS; ++c) L[c] = __shfl_up_sync(FULL, P[c], 1, N);
            roe_flux_prim_fp64(L, P, n0x, n1x, fx);
#pragma unroll
            for (int f = 0; f < 4; ++f) fxr[f] = __shfl_down_sync(FULL, fx[f], 1, N);
            double r[4] = {0.0, 0.0, 0.0, 0.0};
            edge_sum(j, r);
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                if (i > 0) r[f] = r[f] - fx[f];
                if (i < N - 1) r[f] = r[f] + fxr[f];
                if (has_fy) r[f] = r[f] - fy[f];
                part[f] = r[f];
                qbelow[f] = q4[f];
            }
#pragma unroll
            for (int c = 0; c < RS; ++c) below[c] = P[c];
        }
        {
            // the half's top row: the face between rows R-1 and R (h = 0) or
            // the patch's top edge, already summed (h = 1)
            double a0r[4];
            load_a0(R * h + R - 1, a0r);
            finish(R * h + R - 1, h == 0 ? smid[w][sub][i] : nullptr, a0r);
        }
        __syncwarp();  // the next item rewrites this warp's tables
        unsigned nxt = 0;
        if (lane == 0) nxt = atomicAdd(&a.scal->work_next, 1u);
        item = nwarps + (int)__shfl_sync(FULL, nxt, 0);
    }

    sweep_reduce<WARPS>(a, my_dt_min, my_norm, my_flags, red, &s_last);
}

template <int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) sweep64_16_kernel(const StageArgs a)
{
    sweep64_body<16, WARPS>(a);
}

template <int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) sweep64_8_kernel(const StageArgs a)
{
    sweep64_body<8, WARPS>(a);
}

}  // namespace amrgpu
