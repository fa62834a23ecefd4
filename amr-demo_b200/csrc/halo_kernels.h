// halo_kernels.h -- host launchers of halo.cu (ghost-quad pack / unpack).
#pragma once

#include <cuda_runtime.h>

namespace amrgpu {

// out[k] = record of local quad list[k] (4 fields x n*n doubles), k < count
cudaError_t launch_halo_pack(const double *q, long long stride, int n, const int *list, int count, double *out,
                             int sms, cudaStream_t st);
// quad first_quad + k <- in[k], k < count
cudaError_t launch_halo_unpack(double *q, long long stride, int n, int first_quad, int count, const double *in,
                               int sms, cudaStream_t st);
// The same in the edge-strip format (16*n doubles per quad: per field the
// n cells of sides 0, 1, 2, 3); unpack writes only the ghosts' edge cells.
cudaError_t launch_halo_pack_edges(const double *q, long long stride, int n, const int *list, int count,
                                   double *out, int sms, cudaStream_t st);
cudaError_t launch_halo_unpack_edges(double *q, long long stride, int n, int first_quad, int count,
                                     const double *in, int sms, cudaStream_t st);

}  // namespace amrgpu
