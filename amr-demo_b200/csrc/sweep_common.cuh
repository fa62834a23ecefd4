// sweep_common.cuh -- the parts every row-sweep stage kernel shares: the
// step size of the stage (and, on a step's last stage, the advance of the
// step scalars), and the block reductions after the sweep (CFL minimum,
// residual norm in a fixed order, error flags, reset of the quad counter).
#pragma once

#include "device_common.cuh"
#include "stage_kernel.cuh"

namespace amrgpu {

// dt of this step from slot a.slot_read (the cap when the CFL step is off,
// the reference's RK2), clipped at the final time; the last stage of a step
// (block 0, thread 0) advances the time, counts the step and re-arms the
// slots for the next steps.
__device__ __forceinline__ double sweep_step_dt(const StageArgs &a)
{
    const StepSlot slot = a.scal->slot[a.slot_read];
    double dt = __longlong_as_double((long long)slot.dt_bits);
    if (!a.cfl_on) dt = a.dt_cap;
    if (a.final_time > 0.0) {
        double rem = a.final_time - slot.time;
        if (rem < dt) dt = rem;
        if (dt < 0.0) dt = 0.0;
    }
    if (a.last_stage && blockIdx.x == 0 && threadIdx.x == 0) {
        a.scal->slot[a.slot_write].time = slot.time + dt;
        a.scal->dt_used = dt;
        if (dt > 0.0) a.scal->steps += 1;
        a.scal->slot[a.slot_reset].dt_bits = (unsigned long long)__double_as_longlong(a.dt_cap);
        if (!a.cfl_on)
            a.scal->slot[a.slot_write].dt_bits = (unsigned long long)__double_as_longlong(a.dt_cap);
    }
    return dt;
}

// After the sweep: the CFL minimum (one 64-bit atomicMin per block on the
// order-preserving image of the positive double), the norm partials summed
// by the last block to finish in a fixed order (strided per thread, then
// warp and block trees, so the result does not depend on scheduling), the
// error flags; the last block also resets the quad counter and the block
// ticket for the next launch. red holds 64 doubles, s_last one int, both in
// shared memory.
template <int WARPS>
__device__ __forceinline__ void sweep_reduce(const StageArgs &a, double my_dt_min, double my_norm, int my_flags,
                                             double *red, int *s_last)
{
    constexpr unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    int wflags = __reduce_or_sync(FULL, my_flags);
    if (wflags && lane == 0) atomicOr(&a.scal->flags, wflags);
    if (a.last_stage) {
        double wmin = warp_min(my_dt_min);
        double wsum = warp_sum(my_norm);
        if (lane == 0) { red[w] = wmin; red[32 + w] = wsum; }
    }
    __syncthreads();
    if (tid == 0) {
        if (a.last_stage) {
            double bmin = red[0], bsum = red[32];
            for (int k = 1; k < WARPS; ++k) {
                bmin = (red[k] < bmin) ? red[k] : bmin;
                bsum += red[32 + k];
            }
            if (a.cfl_on)
                atomicMin(&a.scal->slot[a.slot_write].dt_bits, (unsigned long long)__double_as_longlong(bmin));
            a.partials[blockIdx.x] = bsum;
        }
        __threadfence();
        const unsigned ticket = atomicAdd(&a.scal->done_blocks, 1u);
        *s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!*s_last) return;
    __threadfence();
    if (a.last_stage) {
        double part = 0.0;
        for (int b = tid; b < (int)gridDim.x; b += WARPS * 32) part += __ldcg(a.partials + b);
        part = warp_sum(part);
        if (lane == 0) red[w] = part;
        __syncthreads();
        if (tid == 0) {
            double tot = red[0];
            for (int k = 1; k < WARPS; ++k) tot += red[k];
            a.scal->norm_sq = tot;
            if (!isfinite(tot)) atomicOr(&a.scal->flags, kFlagNonFinite);
        }
    }
    if (tid == 0) {
        a.scal->work_next = 0u;
        a.scal->done_blocks = 0u;
    }
}

}  // namespace amrgpu
