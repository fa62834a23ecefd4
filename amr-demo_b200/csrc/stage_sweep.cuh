// stage_sweep.cuh -- the FP32-flux form's RK stage for 16x16 and 8x8
// patches as a row sweep: one warp per 16x16 quadrant (two per warp for
// 8x8), no shared-memory records and no block-wide barriers between phases.
//
// Same arithmetic as stage_kernel<16, ..., FP32> (the reference's
// flux_roe_2d, flux_2d_module.F90:63-182, and boundary flux, bc_2d_module.F90,
// in FP32 on per-cell records; FP64 residual sums, stage update, norm and
// conservation; FP32 CFL candidate), reorganised for the register file:
//
//   lane = (sub, h, i): quad sub of the warp's 32/(2N) quads, column
//        i < N of the patch, rows R*h .. R*h+R-1 with R = N/2 (for 16x16:
//        one quad, i = lane & 15, rows 8h .. 8h+7).
//   edges   per quad, the 4 x 16 edge faces (each lane one per round: the
//           own edge cell's record, the neighbour cell(s) the reference
//           pairs it with, the Roe or boundary flux, a coarse hanging edge's
//           two fluxes summed in FP64) and the N faces between rows R-1 and R
//           go to a small per-warp table, in the interior sign convention
//           (a cell adds -F at its low face and +F at its high face);
//   sweep   R steps; at step t lane (i, h) loads cell (i, Rh+t) straight
//           from HBM (N lanes read 8N contiguous bytes per field), builds
//           its record in registers, and evaluates the x-face flux at i-1/2
//           (the left neighbour's record taken by a warp shuffle) and the
//           y-face flux at j-1/2 (the record it kept of the row below)
//           together, one face per half of sm_100's paired FP32
//           instructions; it hands the x-face flux to lane i-1 (which needs
//           it as its i+1/2 face) by a second shuffle. Row j-1 is then
//           complete: -F(x-1/2) +F(x+1/2)
//           -F(y-1/2) +F(y+1/2), summed in FP64, divided by the volume,
//           negated, and the stage update is written.
//
// Per cell-stage this is about 1.1 (packed) flux evaluations, one record,
// 12 shuffles and the update: no per-face index decoding, no record stores
// and reloads, no barrier between the record, face and cell phases.
#pragma once

#include <type_traits>

#include "async_copy.cuh"
#include "flux_fp32.cuh"
#include "stage_kernel.cuh"
#include "sweep_common.cuh"

namespace amrgpu {

// a where the mask is all ones, b where it is zero: a select by bitwise
// operations, which the compiler cannot turn into a branch
__device__ __forceinline__ double blend_d(unsigned long long mask, double a, double b)
{
    const unsigned long long x = (unsigned long long)__double_as_longlong(a);
    const unsigned long long y = (unsigned long long)__double_as_longlong(b);
    return __longlong_as_double((long long)((x & mask) | (y & ~mask)));
}

// Neighbour cell facing position p of side s (the cell on the neighbour's
// opposite side) in a patch of run-time size n.
__device__ __forceinline__ int facing_cell_rt(int s, int p, int n)
{
    if (s == 0) return p * n + (n - 1);
    if (s == 1) return p * n;
    if (s == 2) return (n - 1) * n + p;
    return p;
}

// Per-warp scalars of the sweep's block reductions.
struct SweepAcc {
    double dt_min;
    double norm;
    int flags;
};

// One work item of the row sweep: the warp's QPW quads, this lane's quad
// `quad` (computed but neither stored nor reduced when !valid). sedge is the
// warp's edge table, [quad of the warp][side 0..3, 4 = faces between rows
// R-1 and R][position][field].
//
// MIXED: the mesh holds 8x8 and 16x16 quads (extension, no reference
// counterpart): the quad's state starts at mix[quad].base, and an edge whose
// neighbour has another patch size pairs cells by position along the edge.
// The edge is cut into pieces of the finer side's cell length; each piece
// pairs the own cell and the neighbour cell that cover it, and its flux
// (normal length = the finer cell length) goes to both, evaluated by each
// quad from the same two records at the same call site, so the pair sees
// the same bits (exact conservation). A coarser own cell sums its pieces in
// FP64 in edge order, as a coarse hanging edge sums its two fluxes. Sides
// whose neighbour has this quad's patch size keep the reference's pairing
// (physics_residual_face_*_structured.c: the same position, a coarse
// hanging edge's two index-paired fluxes).
template <int N, bool MIXED, int SO = 0>
__device__ __forceinline__ void sweep_quad(const StageArgs &a, double (*sedge)[5][N][4], double *sa0, int quad,
                                           bool valid, int lane, double dt, const float qinf[4], SweepAcc &acc,
                                           unsigned &next_claim)
{
    static_assert(N == 16 || N == 8, "row sweep for 16x16 and 8x8 patches");
    constexpr int NN = N * N;
    constexpr int R = N / 2;           // rows per half-patch
    constexpr unsigned FULL = 0xffffffffu;
    const int sub = lane / (2 * N), l = lane % (2 * N);
    const int i = l % N, h = l / N;
    const long long stride = a.stride;
    double &my_dt_min = acc.dt_min;
    double &my_norm = acc.norm;
    int &my_flags = acc.flags;
    {
        const QuadDesc &qd = a.quads[quad];
        const double *g = qd.corner;
        const double hx = (g[2] - g[0]) / (double)N, hy = (g[5] - g[1]) / (double)N;
        const double vol = hx * hy, inv_vol = 1.0 / (hx * hy);
        const float fhx = (float)hx, fhy = (float)hy;
        const long long qbase = MIXED ? (long long)a.mix[quad].base : (long long)quad * NN;
        const double *Qq = a.qin + qbase;

        // ---------------- edges: round 0 sides 0 / 1, round 1 sides 2 / 3
        // A side as this lane sees it: its own edge cell, the pieces its edge
        // cell pairs with (one for a full or fine side, two for a coarse
        // hanging side, by position along the edge when the neighbour's
        // patch size differs) and the face normal's length.
        struct EdgeSide {
            SideDesc d;
            int s, own, nk, nn, ratio, hang_half;
            long long nb0, nb1;
            float hc, hp;
        };
        auto side_info = [&](int round) {
            EdgeSide e;
            e.s = 2 * round + h;
            e.d = qd.side[e.s];
            const int m = i;
            e.own = (e.s == 0) ? m * N : (e.s == 1) ? m * N + N - 1 : (e.s == 2) ? m : (N - 1) * N + m;
            e.hc = (float)cell_h_of(a.h_base, e.d.level, N);
            e.hp = e.hc;
            e.nk = (e.d.kind == kSideCoarseHang) ? 2 : 1;
            e.nn = N;
            e.ratio = 0;
            e.hang_half = 0;
            e.nb0 = e.nb1 = 0;
            if constexpr (MIXED) {
                if (e.d.kind != kSideBoundary) {
                    const MixSide ms = a.mix[quad].side[e.s];
                    e.nb0 = ms.base0;
                    e.nb1 = ms.base1;
                    if (ms.n != N) {
                        e.nn = ms.n;
                        e.hang_half = ms.half;
                        double hn;
                        if (e.d.kind == kSideFull) {
                            e.ratio = e.nn > N ? e.nn / N : 1;
                            hn = cell_h_of(a.h_base, e.d.level, e.nn);
                            e.hp = (float)fmin(cell_h_of(a.h_base, e.d.level, N), hn);
                        } else if (e.d.kind == kSideCoarseHang) {
                            e.ratio = 2 * e.nn >= N ? 2 * e.nn / N : 1;
                            hn = cell_h_of(a.h_base, e.d.level, e.nn);
                            e.hp = (float)fmin(cell_h_of(a.h_base, e.d.level - 1, N), hn);
                        } else {
                            e.ratio = 1;
                            hn = cell_h_of(a.h_base, e.d.level - 1, e.nn);
                            e.hp = (float)fmin(cell_h_of(a.h_base, e.d.level, N), hn);
                        }
                        e.nk = e.ratio;
                    }
                }
            }
            return e;
        };
        // state offset (first cell of the quad) and cell of piece k
        auto piece_src = [&](const EdgeSide &e, int k, long long &nb, int &fc) {
            const int m = i;
            if constexpr (MIXED) nb = k == 0 ? e.nb0 : e.nb1;
            else nb = (long long)(k == 0 ? e.d.nbr0 : e.d.nbr1) * NN;
            fc = facing_cell<N>(e.s, m);
            if (MIXED && e.ratio > 0) {
                // geometric pairing with a neighbour of another size
                int p, which = 0;
                if (e.d.kind == kSideFull) {
                    p = e.nn > N ? m * e.ratio + k : m * e.nn / N;
                } else if (e.d.kind == kSideCoarseHang) {
                    const int gp = 2 * e.nn >= N ? m * e.ratio + k : m * 2 * e.nn / N;
                    which = (gp / e.nn) ^ e.hang_half;
                    p = gp % e.nn;
                } else {
                    p = (e.hang_half * N + m) * e.nn / (2 * N);
                }
                nb = which ? e.nb1 : e.nb0;
                fc = facing_cell_rt(e.s, p, e.nn);
            }
        };
        // every load of the edge phase first, so that their latencies
        // overlap instead of following one another: the quad's own cells
        // (both rounds' edge cells, the rows R-1 / R, the sweep's first row)
        // need no descriptor and go out at once; the first neighbour cell of
        // each round follows its side descriptor
        double qo[2][4], qn0[2][4], qmid[4], qnext[4];
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            const int s = 2 * round + h, m = i;
            const int own = (s == 0) ? m * N : (s == 1) ? m * N + N - 1 : (s == 2) ? m : (N - 1) * N + m;
#pragma unroll
            for (int f = 0; f < 4; ++f) qo[round][f] = Qq[f * stride + own];
        }
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            qmid[f] = Qq[f * stride + (R - 1 + h) * N + i];
            qnext[f] = Qq[f * stride + (R * h) * N + i];
        }
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            const EdgeSide e = side_info(round);
            long long nb = qbase;
            int fc = e.own;  // a boundary side reads its own cell again (unused)
            if (e.d.kind != kSideBoundary) piece_src(e, 0, nb, fc);
#pragma unroll
            for (int f = 0; f < 4; ++f) qn0[round][f] = a.qin[nb + f * stride + fc];
        }
#pragma unroll
        for (int round = 0; round < 2; ++round) {
            const EdgeSide e = side_info(round);
            const int s = e.s, m = i;
            float Po[8], fl[4];
            cell_prims_fp32(qo[round], Po);
            double E[4];
            if (e.d.kind == kSideBoundary) {
                const float n0 = round == 0 ? (s == 0 ? -e.hc : e.hc) : 0.0f;
                const float n1 = round == 0 ? 0.0f : (s == 2 ? -e.hc : e.hc);
                bc_flux_rec_fp32(e.d.bc, Po, n0, n1, qinf, fl);
#pragma unroll
                for (int f = 0; f < 4; ++f) E[f] = (s & 1) ? (double)fl[f] : -(double)fl[f];
            } else {
                // one flux site for a side's one or two neighbours: the
                // neighbour quad computes the same face at the same site, so
                // both see bit-identical values (conservation)
                auto piece_flux = [&](const double qn4[4]) {
                    float Pn[8];
                    cell_prims_fp32(qn4, Pn);
                    const float *L = (s & 1) ? Po : Pn;
                    const float *R = (s & 1) ? Pn : Po;
                    if (round == 0) roe_flux_axis_fp32<0>(L, R, e.hp, fl);
                    else roe_flux_axis_fp32<1>(L, R, e.hp, fl);
                };
                piece_flux(qn0[round]);
#pragma unroll
                for (int f = 0; f < 4; ++f) E[f] = 0.0 + (double)fl[f];
#pragma unroll 1
                for (int k = 1; k < e.nk; ++k) {
                    long long nb;
                    int fc;
                    piece_src(e, k, nb, fc);
                    double qn4[4];
#pragma unroll
                    for (int f = 0; f < 4; ++f) qn4[f] = a.qin[nb + f * stride + fc];
                    piece_flux(qn4);
#pragma unroll
                    for (int f = 0; f < 4; ++f) E[f] = E[f] + (double)fl[f];
                }
            }
#pragma unroll
            for (int f = 0; f < 4; ++f) sedge[sub][s][m][f] = E[f];
        }
        // ---------------- the faces between rows R-1 and R (column i)
        {
            float P[8], O[8], fl[4];
            cell_prims_fp32(qmid, P);
#pragma unroll
            for (int k = 0; k < 8; ++k) O[k] = __shfl_xor_sync(FULL, P[k], N);
            if (h == 0) {
                roe_flux_axis_fp32<1>(P, O, fhx, fl);
#pragma unroll
                for (int f = 0; f < 4; ++f) sedge[sub][4][i][f] = (double)fl[f];
            }
        }
        __syncwarp();

        // ---------------- sweep over the lane's R rows
        float below[8];      // record of the row below (y-face partner)
        double part[4];      // (-F(x-1/2) + F(x+1/2)) - F(y-1/2) of the row below
        double qbelow[4];    // input state of the row below
        // the stage's first auxiliary input (Q0 of the Shu-Osher stages 2-3)
        // of row j goes by cp.async into this lane's slot j & 1 of the warp's
        // buffer sa0 ([slot][field][lane]) while row j is swept, and is read
        // when row j is finished in the next step: prefetched a row ahead
        // without holding it in registers
        const bool has_a0 = SO > 0 ? SO >= 2 : a.a0 != nullptr;
        auto finish = [&](int jr, const double gup[4]) {
            const long long gi = qbase + jr * N + i;
            double kv[4], qn[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                const double r = part[f] + gup[f];
                kv[f] = -(r * inv_vol);
            }
            if (!valid) return;
            auto A0 = [&](int f) -> double { return has_a0 ? sa0[(jr & 1) * 128 + f * 32 + lane] : 0.0; };
            auto A1 = [&](int f) -> double { return a.a1[f * stride + gi]; };
            if constexpr (SO > 0) rk_update<kSchemeRK3ShuOsher, SO>(a, dt, stride, gi, qbelow, kv, A0, A1, qn);
            else rk_update(a, dt, stride, gi, qbelow, kv, A0, A1, qn);
            if (SO > 0 ? SO == 3 : a.last_stage != 0) {
#pragma unroll
                for (int f = 0; f < 4; ++f) my_norm += kv[f] * kv[f];
                if (a.cfl_on) {
                    const double cand = cfl_candidate_fp32(qn, vol, a.cfl);
                    if (cand < my_dt_min) my_dt_min = cand;
                }
                const double rho = qn[0];
                const double pe = qn[3] * rho - 0.5 * (qn[1] * qn[1] + qn[2] * qn[2]);
                if (!(rho > 0.0) || !(pe > 0.0)) my_flags |= kFlagNegative;
            }
        };
        // lanes whose low / high x-face is an edge face: all-ones masks
        const unsigned long long m_lo = i == 0 ? ~0ull : 0ull, m_hi = i == N - 1 ? ~0ull : 0ull;
        // one row step. The first row (its y-face below is an edge or the row
        // R-1/R face, no row below to finish) and the last (no row above to
        // prefetch) are separate copies, so the loop in between tests neither.
        auto row = [&](int t, auto first_c, auto last_c) {
            constexpr bool FIRST = decltype(first_c)::value;
            constexpr bool LAST = decltype(last_c)::value;
            const int j = R * h + t;
            double q4[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) q4[f] = qnext[f];
            if constexpr (!LAST) {
#pragma unroll
                for (int f = 0; f < 4; ++f) qnext[f] = Qq[f * stride + (j + 1) * N + i];
            } else {
                // the warp's next work item is claimed a row before this one
                // ends: the atomic's round trip overlaps the last row
                if (lane == 0) next_claim = atomicAdd(&a.scal->work_next, 1u);
            }
            // the auxiliary input of this row, used when the row is finished
            // in the next step (its latency is covered by the fluxes)
            if (has_a0) {
#pragma unroll
                for (int f = 0; f < 4; ++f)
                    cp_async8(sa0 + (j & 1) * 128 + f * 32 + lane, a.a0 + f * stride + qbase + j * N + i);
                cp_async_commit();
            }
            float P[8];
            cell_prims_fp32(q4, P);
            // the x-face at i-1/2 (lane 0's left face is an edge face) and
            // the y-face at j-1/2 in one packed evaluation (the first row's
            // y-face is an edge or the row R-1/R face: its half is unused)
            float L[8], fx[4], fy[4], fxr[4];
#pragma unroll
            for (int k = 0; k < 8; ++k) L[k] = __shfl_up_sync(FULL, P[k], 1, N);
            if constexpr (FIRST) {
#pragma unroll
                for (int k = 0; k < 8; ++k) below[k] = P[k];
            }
            roe_flux_axis_pair_fp32(L, below, P, fhy, fhx, fx, fy);
#pragma unroll
            for (int f = 0; f < 4; ++f) fxr[f] = __shfl_down_sync(FULL, fx[f], 1, N);
            double xp[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                // every lane reads the edge faces (one address per half) and
                // converts its interior ones; the choice is a bitwise blend
                const double el = sedge[sub][0][j][f], er = sedge[sub][1][j][f];
                const double fl = blend_d(m_lo, el, (double)fx[f]);
                const double fr = blend_d(m_hi, er, (double)fxr[f]);
                xp[f] = fr - fl;
            }
            // y-face at j-1/2 (the first row's is an edge or the row R-1/R face)
            double gy[4];
            if constexpr (FIRST) {
                const double *ge = h == 0 ? sedge[sub][2][i] : sedge[sub][4][i];
#pragma unroll
                for (int f = 0; f < 4; ++f) gy[f] = ge[f];
            } else {
#pragma unroll
                for (int f = 0; f < 4; ++f) gy[f] = (double)fy[f];
                if (has_a0) cp_async_wait_group<1>();  // row j-1's input has landed
                finish(j - 1, gy);
            }
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                part[f] = xp[f] - gy[f];
                qbelow[f] = q4[f];
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) below[k] = P[k];
        };
        row(0, std::true_type{}, std::false_type{});
#pragma unroll 1
        for (int t = 1; t < R - 1; ++t) row(t, std::false_type{}, std::false_type{});
        row(R - 1, std::false_type{}, std::true_type{});
        {
            double gtop[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) gtop[f] = h == 0 ? sedge[sub][4][i][f] : sedge[sub][3][i][f];
            if (has_a0) cp_async_wait_group<0>();
            finish(R * h + R - 1, gtop);
        }
        __syncwarp();  // the next item rewrites this warp's edge table
    }
}

// The uniform-size row sweep. Work items (QPW consecutive quads each): each
// warp's first one by its index, then the next free one from a counter
// (work_next, reset to 0 by the last block; claimed during an item's last
// row), so that warps and SMs that finish early take more and the tail
// stays short. A quad past the end (odd
// count, 8x8) is computed on its item's first quad and neither stored nor
// reduced.
template <int N, int WARPS, int SO>
__device__ __forceinline__ void sweep_body(const StageArgs &a)
{
    constexpr int QPW = 32 / (2 * N);
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ double sedge[WARPS][QPW][5][N][4];
    __shared__ __align__(16) double sa0[WARPS][2 * 4 * 32];
    __shared__ double red[64];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sub = lane / (2 * N);
    const double dt = sweep_step_dt(a);
    const float qinf[4] = {(float)a.qinflow[0], (float)a.qinflow[1], (float)a.qinflow[2], (float)a.qinflow[3]};
    SweepAcc acc{a.dt_cap, 0.0, 0};
    const int nwarps = gridDim.x * WARPS;
    const int nitems = (a.nquad + QPW - 1) / QPW;
    int item = blockIdx.x * WARPS + w;
    while (item < nitems) {
        const bool valid = QPW == 1 || item * QPW + sub < a.nquad;
        const int quad = valid ? item * QPW + sub : item * QPW;
        unsigned nxt = 0;  // claimed by lane 0 during the item's last row
        sweep_quad<N, false, SO>(a, sedge[w], sa0[w], quad, valid, lane, dt, qinf, acc, nxt);
        item = nwarps + (int)__shfl_sync(FULL, nxt, 0);
    }
    sweep_reduce<WARPS>(a, acc.dt_min, acc.norm, acc.flags, red, &s_last);
}

// The mixed-size row sweep: one launch over a work list of the 16x16 quads
// (one item each) followed by the 8x8 quads (two per item), claimed from
// one counter as above; an item's patch size decides which body runs (the
// choice is uniform over the warp). The two bodies share one per-warp edge
// table (320 doubles for either size).
template <int WARPS, int SO>
__device__ __forceinline__ void sweep_body_mixed(const StageArgs &a)
{
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ double sedge_raw[WARPS][5 * 16 * 4];
    __shared__ __align__(16) double sa0[WARPS][2 * 4 * 32];
    __shared__ double red[64];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const double dt = sweep_step_dt(a);
    const float qinf[4] = {(float)a.qinflow[0], (float)a.qinflow[1], (float)a.qinflow[2], (float)a.qinflow[3]};
    SweepAcc acc{a.dt_cap, 0.0, 0};
    const int nwarps = gridDim.x * WARPS;
    const int nitems = a.nwork16 + (a.nwork8 + 1) / 2;
    int item = blockIdx.x * WARPS + w;
    while (item < nitems) {
        unsigned nxt = 0;  // claimed by lane 0 during the item's last row
        if (item < a.nwork16) {
            sweep_quad<16, true, SO>(a, reinterpret_cast<double(*)[5][16][4]>(sedge_raw[w]), sa0[w], a.work[item],
                                     true, lane, dt, qinf, acc, nxt);
        } else {
            const int k = 2 * (item - a.nwork16) + lane / 16;
            const bool valid = k < a.nwork8;
            const int quad = a.work[a.nwork16 + (valid ? k : k - 1)];
            sweep_quad<8, true, SO>(a, reinterpret_cast<double(*)[5][8][4]>(sedge_raw[w]), sa0[w], quad, valid,
                                    lane, dt, qinf, acc, nxt);
        }
        item = nwarps + (int)__shfl_sync(FULL, nxt, 0);
    }
    sweep_reduce<WARPS>(a, acc.dt_min, acc.norm, acc.flags, red, &s_last);
}

// SO = 0: any scheme and stage, read from the arguments; SO = 1..3: stage
// SO of the Shu-Osher RK3 (the FP32-flux form's scheme) fixed at compile
// time, so the row loop carries no per-cell scheme or stage test.
template <int WARPS, int MINB, int SO = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB) sweep16_kernel(const StageArgs a)
{
    stage_launch_gate();
    sweep_body<16, WARPS, SO>(a);
}

template <int WARPS, int MINB, int SO = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB) sweep8_kernel(const StageArgs a)
{
    stage_launch_gate();
    sweep_body<8, WARPS, SO>(a);
}

template <int WARPS, int MINB, int SO = 0>
__global__ void __launch_bounds__(WARPS * 32, MINB) sweep_mixed_kernel(const StageArgs a)
{
    stage_launch_gate();
    sweep_body_mixed<WARPS, SO>(a);
}

}  // namespace amrgpu
