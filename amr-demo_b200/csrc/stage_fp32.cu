// stage_fp32.cu -- FP32-flux instantiations of the stage kernel: face
// fluxes, normals, boundary states and the CFL candidate in FP32; the
// conserved state, the per-cell residual sums (hanging-face corrections
// included), the division by the volume and the stage update stay in FP64.
#include <cuda_runtime.h>

#include "flux_fp32.cuh"
#include "flux_fp64.cuh"
#include "launch_table.h"
#include "remap_cfl.cuh"
#include "stage_kernel.cuh"
#include "stage_sweep.cuh"

namespace amrgpu {

struct FluxOpsFP32 {
    __device__ static __forceinline__ void prims(const double *q, float *P) { cell_prims_fp32(q, P); }
    __device__ static __forceinline__ void roe(const float *l, const float *r, float n0, float n1,
                                               float *f)
    {
        roe_flux_prim_fp32(l, r, n0, n1, f);
    }
    // axis-aligned face with positive normal: n0 = h (DIR 0) or n1 = h (DIR 1)
    template <int DIR>
    __device__ static __forceinline__ void roe_axis(const float *l, const float *r, float n0, float n1,
                                                    float *f)
    {
        roe_flux_axis_fp32<DIR>(l, r, DIR == 0 ? n0 : n1, f);
    }
    __device__ static __forceinline__ void bc(int bc, const float *q, float n0, float n1,
                                              const float *qin, float *f)
    {
        bc_flux_rec_fp32(bc, q, n0, n1, qin, f);
    }
    __device__ static __forceinline__ double cfl(const double *q, double vol, double c)
    {
        return cfl_candidate_fp32(q, vol, c);
    }
};

// CFL step of a state for the FP32-flux form (segment prologue): the same
// candidate and rectangle volume as the stage kernel's last stage, so a step
// takes the same dt whether or not it starts a segment.
template <int N>
__global__ void __launch_bounds__(256) cfl_kernel_f32(const CflArgs a)
{
    constexpr int NN = N * N;
    __shared__ double red[8];
    double best = __longlong_as_double((long long)a.scal->slot[a.slot].dt_bits);
    const long long ncells = (long long)a.nquad * NN;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(c / NN);
        const double *g = a.quads[q].corner;
        const double hx = (g[2] - g[0]) / (double)N, hy = (g[5] - g[1]) / (double)N;
        double q4[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) q4[f] = a.qin[f * a.stride + c];
        const double cand = cfl_candidate_fp32(q4, hx * hy, a.cfl);
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

// cfl_kernel_f32's candidate of one cell from its values, for
// remap_cfl_kernel
struct CflCandFP32 {
    template <int N>
    __device__ static __forceinline__ double candidate(const CflArgs &a, int q, int, const double q4[4])
    {
        const double *g = a.quads[q].corner;
        const double hx = (g[2] - g[0]) / (double)N, hy = (g[5] - g[1]) / (double)N;
        return cfl_candidate_fp32(q4, hx * hy, a.cfl);
    }
};

const void *remap_cfl_kernel_fp32(int n)
{
    switch (n) {
    case 2: return (const void *)remap_cfl_kernel<2, CflCandFP32>;
    case 4: return (const void *)remap_cfl_kernel<4, CflCandFP32>;
    case 8: return (const void *)remap_cfl_kernel<8, CflCandFP32>;
    case 16: return (const void *)remap_cfl_kernel<16, CflCandFP32>;
    default: return nullptr;
    }
}

const void *cfl_kernel_fp32(int n)
{
    switch (n) {
    case 2: return (const void *)cfl_kernel_f32<2>;
    case 4: return (const void *)cfl_kernel_f32<4>;
    case 8: return (const void *)cfl_kernel_f32<8>;
    case 16: return (const void *)cfl_kernel_f32<16>;
    default: return nullptr;
    }
}

#define AMRGPU_STAGE32(N, QPB, T, MINB)                                                        \
    StageLaunch{N, QPB, T, MINB, StageSmem<N, QPB, true>::total,                               \
                (const void *)stage_kernel<N, QPB, T, MINB, true, FluxOpsFP32>}

// row-sweep kernel for 16x16 patches: one warp per quad, "quads per
// block" = warps per block, no dynamic shared memory; all at 128
// registers (16 resident warps per SM): fewer registers spill and run slower
#define AMRGPU_SWEEP16(W, MINB)                                                                          \
    StageLaunch{16, W, 32 * (W), MINB, 0, (const void *)sweep16_kernel<W, MINB>, 1,                      \
                {(const void *)sweep16_kernel<W, MINB, 1>, (const void *)sweep16_kernel<W, MINB, 2>,     \
                 (const void *)sweep16_kernel<W, MINB, 3>},                                               \
                kSchemeRK3ShuOsher}
#define AMRGPU_SWEEP8(W, MINB)                                                                           \
    StageLaunch{8, 2 * (W), 32 * (W), MINB, 0, (const void *)sweep8_kernel<W, MINB>, 1,                  \
                {(const void *)sweep8_kernel<W, MINB, 1>, (const void *)sweep8_kernel<W, MINB, 2>,       \
                 (const void *)sweep8_kernel<W, MINB, 3>},                                                \
                kSchemeRK3ShuOsher}
#define AMRGPU_SWEEPMIX(W, MINB)                                                                         \
    StageLaunch{0, W, 32 * (W), MINB, 0, (const void *)sweep_mixed_kernel<W, MINB>, 1,                   \
                {(const void *)sweep_mixed_kernel<W, MINB, 1>, (const void *)sweep_mixed_kernel<W, MINB, 2>, \
                 (const void *)sweep_mixed_kernel<W, MINB, 3>},                                            \
                kSchemeRK3ShuOsher}

static const StageLaunch kTable32[] = {
    AMRGPU_SWEEP16(4, 4),   // 128 registers, 16 warps per SM
    AMRGPU_SWEEP16(2, 8),
    AMRGPU_SWEEP16(8, 2),
    AMRGPU_STAGE32(16, 1, 288, 3),
    AMRGPU_STAGE32(16, 1, 288, 2),
    AMRGPU_STAGE32(16, 2, 544, 1),
    AMRGPU_STAGE32(16, 2, 576, 1),
    AMRGPU_STAGE32(16, 1, 544, 2),
    AMRGPU_SWEEP8(4, 4),    // two 8x8 quads per warp
    AMRGPU_SWEEP8(2, 8),
    AMRGPU_SWEEP8(8, 2),
    AMRGPU_STAGE32(8, 4, 288, 3),
    AMRGPU_STAGE32(8, 2, 160, 4),
    AMRGPU_STAGE32(8, 8, 576, 1),
    AMRGPU_STAGE32(4, 8, 160, 4),
    AMRGPU_STAGE32(4, 16, 320, 2),
    AMRGPU_STAGE32(2, 16, 96, 4),
    AMRGPU_STAGE32(2, 32, 192, 2),
};

int stage_table_fp32(const StageLaunch **out)
{
    *out = kTable32;
    return int(sizeof(kTable32) / sizeof(kTable32[0]));
}

// The mixed-size sweep's shapes (n = 0): two warps per block at 128
// registers (16 warps per SM; the two bodies spill ~100 bytes there), and at
// 159 registers without spills (12 warps per SM). Every shape gives the same
// bits; the autotuner picks one per mesh-size bucket.
static const StageLaunch kMixed[] = {
    AMRGPU_SWEEPMIX(2, 8),
    AMRGPU_SWEEPMIX(2, 6),
    AMRGPU_SWEEPMIX(4, 3),
};

const StageLaunch *stage_launch_mixed() { return &kMixed[0]; }

int stage_table_mixed(const StageLaunch **out)
{
    *out = kMixed;
    return int(sizeof(kMixed) / sizeof(kMixed[0]));
}

}  // namespace amrgpu
