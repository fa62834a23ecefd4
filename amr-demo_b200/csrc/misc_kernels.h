// misc_kernels.h -- host launchers of kernels_misc.cu.
#pragma once

#include <cuda_runtime.h>

namespace amrgpu {

struct QuadDesc;
struct DeviceScalars;

struct TagMethods {
    int method[5];
    double tol[5];
};

cudaError_t launch_aos_to_soa(const double *aos, double *soa, long long ncells, long long stride,
                              cudaStream_t st);
cudaError_t launch_soa_to_aos(const double *soa, double *aos, long long ncells, long long stride,
                              cudaStream_t st);
int totals_grid(long long ncells);
cudaError_t launch_totals(int n, const QuadDesc *quads, const double *q, long long stride, int nquad,
                          double *partials, int grid, cudaStream_t st);
cudaError_t launch_tag(int n, const double *rho, const QuadDesc *quads, int nquad, int nmeth,
                       const TagMethods &m, int *tags, cudaStream_t st);
cudaError_t launch_rearm(DeviceScalars *scal, int slot_now, double cap, cudaStream_t st);
cudaError_t launch_remap(int n, const double *qold, long long stride_old, double *qnew,
                         long long stride_new, const int *kind, const int *src, int nquad_new,
                         cudaStream_t st);

}  // namespace amrgpu
