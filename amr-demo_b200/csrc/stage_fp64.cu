// stage_fp64.cu -- FP64 instantiations of the stage kernel and the CFL
// prologue kernel. This translation unit is compiled with -fmad=false: no
// multiply-add is contracted, so every flux, normal, volume, residual sum
// and stage update is the IEEE-rounded value of the reference's own
// expression, and the plain FP64 form reproduces the reference bit for bit.
#include <cuda_runtime.h>

#include "flux_fp64.cuh"
#include "launch_table.h"
#include "remap_cfl.cuh"
#include "stage_kernel.cuh"
#include "stage_sweep64.cuh"

namespace amrgpu {

struct FluxOpsFP64 {
    __device__ static __forceinline__ void prims(const double *q, double *P) { cell_prims_fp64(q, P); }
    __device__ static __forceinline__ void roe(const double *l, const double *r, double n0, double n1,
                                               double *f)
    {
        roe_flux_prim_fp64(l, r, n0, n1, f);
    }
    // the exact form evaluates every face through the general expression
    template <int DIR>
    __device__ static __forceinline__ void roe_axis(const double *l, const double *r, double n0, double n1,
                                                    double *f)
    {
        roe_flux_prim_fp64(l, r, n0, n1, f);
    }
    __device__ static __forceinline__ void bc(int bc, const double *q, double n0, double n1,
                                              const double *qin, double *f)
    {
        bc_flux_fp64(bc, q, n0, n1, qin, f);
    }
    __device__ static __forceinline__ double cfl(const double *q, double vol, double c)
    {
        return cfl_candidate_fp64(q, vol, c);
    }
};

// solver_time_step_2d_module.F90:26-122 over every cell, folded with the
// cap already in the slot: one warp-shuffle + shared-memory reduction per
// block, one 64-bit atomicMin per block on the order-preserving bit image
// of the (positive) double.
template <int N>
__global__ void __launch_bounds__(256) cfl_kernel(const CflArgs a)
{
    constexpr int NN = N * N;
    __shared__ double red[8];
    const double s = 2.0 / (double)N;
    double best = __longlong_as_double((long long)a.scal->slot[a.slot].dt_bits);
    const long long ncells = (long long)a.nquad * NN;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        int q = (int)(c / NN);
        int r = (int)(c - (long long)q * NN);
        int i = r % N, j = r / N;
        const double *g = a.quads[q].corner;
        double v1 = s * (double)j - 1.0, v2 = s * (double)(j + 1) - 1.0;
        double w1 = s * (double)i - 1.0, w2 = s * (double)(i + 1) - 1.0;
        double x1, y1, x2, y2, x3, y3, x4, y4;
        bilinear_node(g, w1, v1, x1, y1);
        bilinear_node(g, w2, v1, x2, y2);
        bilinear_node(g, w1, v2, x3, y3);
        bilinear_node(g, w2, v2, x4, y4);
        double vol = subcell_volume(x1, y1, x2, y2, x3, y3, x4, y4);
        double q4[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) q4[f] = a.qin[f * a.stride + c];
        double cand = cfl_candidate_fp64(q4, vol, a.cfl);
        if (cand < best) best = cand;
    }
    best = warp_min(best);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = (red[w] < best) ? red[w] : best;
        atomicMin(&a.scal->slot[a.slot].dt_bits, (unsigned long long)__double_as_longlong(best));
    }
}

// cfl_kernel's candidate of one cell from its values (the subcell volume
// from the quad's bilinear corners), for remap_cfl_kernel
struct CflCandFP64 {
    template <int N>
    __device__ static __forceinline__ double candidate(const CflArgs &a, int q, int r, const double q4[4])
    {
        const double s = 2.0 / (double)N;
        const int i = r % N, j = r / N;
        const double *g = a.quads[q].corner;
        double v1 = s * (double)j - 1.0, v2 = s * (double)(j + 1) - 1.0;
        double w1 = s * (double)i - 1.0, w2 = s * (double)(i + 1) - 1.0;
        double x1, y1, x2, y2, x3, y3, x4, y4;
        bilinear_node(g, w1, v1, x1, y1);
        bilinear_node(g, w2, v1, x2, y2);
        bilinear_node(g, w1, v2, x3, y3);
        bilinear_node(g, w2, v2, x4, y4);
        const double vol = subcell_volume(x1, y1, x2, y2, x3, y3, x4, y4);
        return cfl_candidate_fp64(q4, vol, a.cfl);
    }
};

const void *remap_cfl_kernel_fp64(int n)
{
    switch (n) {
    case 2: return (const void *)remap_cfl_kernel<2, CflCandFP64>;
    case 4: return (const void *)remap_cfl_kernel<4, CflCandFP64>;
    case 8: return (const void *)remap_cfl_kernel<8, CflCandFP64>;
    case 16: return (const void *)remap_cfl_kernel<16, CflCandFP64>;
    default: return nullptr;
    }
}

const void *cfl_kernel_fp64(int n)
{
    switch (n) {
    case 2: return (const void *)cfl_kernel<2>;
    case 4: return (const void *)cfl_kernel<4>;
    case 8: return (const void *)cfl_kernel<8>;
    case 16: return (const void *)cfl_kernel<16>;
    default: return nullptr;
    }
}

#define AMRGPU_STAGE64(N, QPB, T, MINB)                                                        \
    StageLaunch{N, QPB, T, MINB, StageSmem<N, QPB, false>::total,                              \
                (const void *)stage_kernel<N, QPB, T, MINB, false, FluxOpsFP64>}

// row-sweep kernels: one warp per 16x16 quad or per two 8x8 quads
#define AMRGPU_SWEEP64_16(W, MINB)                                                                      \
    StageLaunch{16, W, 32 * (W), MINB, Sweep64Smem<16>::bytes(W), (const void *)sweep64_16_kernel<W, MINB>, 1,  \
                {(const void *)sweep64_16_kernel<W, MINB, 1>, (const void *)sweep64_16_kernel<W, MINB, 2>,     \
                 (const void *)sweep64_16_kernel<W, MINB, 3>},                                                 \
                kSchemeRK3}
#define AMRGPU_SWEEP64_8(W, MINB)                                                                       \
    StageLaunch{8, 2 * (W), 32 * (W), MINB, Sweep64Smem<8>::bytes(W), (const void *)sweep64_8_kernel<W, MINB>, 1, \
                {(const void *)sweep64_8_kernel<W, MINB, 1>, (const void *)sweep64_8_kernel<W, MINB, 2>,       \
                 (const void *)sweep64_8_kernel<W, MINB, 3>},                                                  \
                kSchemeRK3}

// Per patch size the first entry is the default launch (a row sweep gives
// way to the size's first block kernel on meshes too small to fill the GPU
// with sweep warps); the autotuner picks among all entries of the size.
static const StageLaunch kTable64[] = {
    AMRGPU_SWEEP64_16(4, 4),  // 128 registers, 16 warps per SM
    AMRGPU_SWEEP64_16(2, 8),
    AMRGPU_SWEEP64_16(4, 3),
    AMRGPU_STAGE64(16, 1, 288, 2),
    AMRGPU_STAGE64(16, 1, 288, 1),
    AMRGPU_STAGE64(16, 2, 576, 1),
    AMRGPU_STAGE64(16, 1, 256, 2),
    AMRGPU_SWEEP64_8(4, 4),   // two 8x8 quads per warp
    AMRGPU_SWEEP64_8(4, 3),
    AMRGPU_STAGE64(8, 4, 288, 2),
    AMRGPU_STAGE64(8, 2, 160, 3),
    AMRGPU_STAGE64(8, 4, 576, 1),
    AMRGPU_STAGE64(4, 8, 160, 3),
    AMRGPU_STAGE64(4, 16, 320, 2),
    AMRGPU_STAGE64(2, 16, 96, 4),
    AMRGPU_STAGE64(2, 32, 192, 2),
};

int stage_table_fp64(const StageLaunch **out)
{
    *out = kTable64;
    return int(sizeof(kTable64) / sizeof(kTable64[0]));
}

}  // namespace amrgpu
