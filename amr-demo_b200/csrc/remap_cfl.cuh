// remap_cfl.cuh -- the state remap of an in-place regrid fused with the
// CFL minimum of the remapped state (the next segment's first dt), in one
// pass over the new mesh's cells instead of two.
//
// The remap is remap_kernel's (kernels_misc.cu): refine injects the parent
// patch into each child (solver_refine_operator_2d.F90:49-52), coarsen
// writes (uc1+uc2+uc3+uc4)*0.25 (solver_coarsen_operator_2d.F90:49-50).
// Each cell's CFL candidate is then taken from the values just written, by
// the candidate functor of the form's CFL prologue kernel (compiled in the
// same translation unit with the same flags), and folded into the step
// slot with the same warp / block minimum and 64-bit atomicMin; the slot
// must hold the dt cap already (rearm_kernel). A minimum does not depend
// on the order, so the dt is the bits the separate kernels give.
#pragma once

#include "stage_kernel.cuh"

namespace amrgpu {

template <int N, class Cand>
__global__ void __launch_bounds__(256) remap_cfl_kernel(const RemapCflArgs a)
{
    constexpr int NN = N * N;
    __shared__ double red[8];
    const CflArgs &c = a.cfl;
    double best = __longlong_as_double((long long)c.scal->slot[c.slot].dt_bits);
    const long long total = (long long)c.nquad * NN;
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < total;
         cell += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(cell / NN);
        const int r = (int)(cell - (long long)q * NN);
        const int s = a.src[q];
        const bool inject = a.kind[q] == 0;
        double v[4];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const double *o = a.qold + f * a.stride_old + r;
            if (inject) {
                v[f] = o[(long long)s * NN];
            } else {
                const double sum = o[(long long)s * NN] + o[(long long)(s + 1) * NN] + o[(long long)(s + 2) * NN] +
                                   o[(long long)(s + 3) * NN];
                v[f] = 0.25 * sum;
            }
            a.qnew[f * c.stride + cell] = v[f];
        }
        const double cand = Cand::template candidate<N>(c, q, r, v);
        if (cand < best) best = cand;
    }
    best = warp_min(best);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = (red[w] < best) ? red[w] : best;
        atomicMin(&c.scal->slot[c.slot].dt_bits, (unsigned long long)__double_as_longlong(best));
    }
}

}  // namespace amrgpu
