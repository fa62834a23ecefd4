// misc_kernels.h -- host launchers of kernels_misc.cu.
#pragma once

#include <cuda_runtime.h>

namespace amrgpu {

struct QuadDesc;
struct MixDesc;
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

// mixed patch sizes (mixed.cu)
struct SizeRule {
    int size[32];  // patch size (8 or 16) of a quad at each level
};
const void *cfl_kernel_mixed();
// Descriptors and work list of a mixed mesh from a forest's leaves (tree,
// level, x, y) and its new quad descriptors: cells / flag16 / base / pos16
// hold nq + 1 ints each; status (3 ints): [0] 1 when a hanging edge's two
// fine quads differ in size, [1] the cells, [2] the 16x16 quads.
size_t build_mix_scan_bytes(int nq);
cudaError_t launch_build_mix(const int4 *leaves, const QuadDesc *quads, int nq, const SizeRule &rule, MixDesc *out,
                             int *work, int *cells, int *flag16, int *base, int *pos16, void *scan_tmp,
                             size_t scan_bytes, int *status, cudaStream_t st);
int totals_mixed_grid(int nquad);
cudaError_t launch_totals_mixed(const QuadDesc *quads, const MixDesc *mix, const double *q, long long stride,
                                int nquad, double *partials, int grid, cudaStream_t st);
cudaError_t launch_tag_mixed(const double *rho, const QuadDesc *quads, const MixDesc *mix, int nquad, int nmeth,
                             const TagMethods &m, int *tags, cudaStream_t st);
cudaError_t launch_remap_mixed(const double *qold, long long stride_old, const MixDesc *mold, double *qnew,
                               long long stride_new, const MixDesc *mnew, const int *kind, const int *src,
                               int nquad_new, cudaStream_t st);

}  // namespace amrgpu
