// stage_fp32.cu -- FP32-flux instantiations of the stage kernel: face
// fluxes, normals and boundary states in FP32; the conserved state, the
// per-cell residual sums (hanging-face corrections included), the division
// by the volume, the stage update and the CFL step stay in FP64.
#include <cuda_runtime.h>

#include "flux_fp32.cuh"
#include "flux_fp64.cuh"
#include "launch_table.h"
#include "stage_kernel.cuh"

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
        return cfl_candidate_fp64(q, vol, c);
    }
};

#define AMRGPU_STAGE32(N, QPB, T, MINB)                                                        \
    StageLaunch{N, QPB, T, MINB, StageSmem<N, QPB, true>::total,                               \
                (const void *)stage_kernel<N, QPB, T, MINB, true, FluxOpsFP32>}

static const StageLaunch kTable32[] = {
    AMRGPU_STAGE32(16, 1, 288, 3),
    AMRGPU_STAGE32(16, 1, 288, 2),
    AMRGPU_STAGE32(16, 2, 544, 1),
    AMRGPU_STAGE32(16, 2, 576, 1),
    AMRGPU_STAGE32(16, 1, 544, 2),
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

}  // namespace amrgpu
