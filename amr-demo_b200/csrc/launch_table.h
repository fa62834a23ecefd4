// launch_table.h -- the compiled stage-kernel variants. Each entry is one
// (patch size n, quads per CTA, threads per CTA) instantiation of
// stage_kernel; the host autotuner times the entries that match a mesh's n
// and keeps the fastest.
#pragma once

#include <cstddef>

namespace amrgpu {

struct StageArgs;

struct StageLaunch {
    int n;
    int qpb;
    int threads;
    int min_blocks;
    size_t smem;
    const void *kernel;  // __global__ void(StageArgs)
    int sweep = 0;       // 1: a row-sweep kernel (one warp per qpb*32/threads quads)
    // the same launch specialised for stages 1..3 of one three-stage scheme
    // (so_scheme: the Shu-Osher RK3 of the FP32-flux form, the reference's
    // RK3 of the FP64 form), when the variant has them
    const void *kernel_so[3] = {nullptr, nullptr, nullptr};
    int so_scheme = -1;
};

int stage_table_fp64(const StageLaunch **out);
int stage_table_fp32(const StageLaunch **out);
// The mixed-size row sweep (8x8 and 16x16 quads in one work list, FP32-flux
// form): n = 0, never a uniform mesh's launch.
const StageLaunch *stage_launch_mixed();
int stage_table_mixed(const StageLaunch **out);

// CFL step of a state (prologue of a segment): min over cells of the
// reference's candidate, folded into scal->slot[slot].dt_bits.
struct CflArgs;
const void *cfl_kernel_fp64(int n);
const void *cfl_kernel_fp32(int n);  // the FP32-flux form's candidate
// The remap of an in-place regrid fused with the CFL minimum of the
// remapped state (remap_cfl.cuh), per form: __global__ void(RemapCflArgs).
const void *remap_cfl_kernel_fp64(int n);
const void *remap_cfl_kernel_fp32(int n);

}  // namespace amrgpu
