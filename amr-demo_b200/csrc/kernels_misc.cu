// kernels_misc.cu -- data-movement and regrid kernels around the stage
// kernel: AoS <-> SoA conversion of the reference's soln array,
// conservation totals, the batched plain refinement indicator and the
// batched refine/coarsen remap.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "misc_kernels.h"
#include "stage_kernel.cuh"

namespace amrgpu {

// reference AoS soln[f + 4*c] (amr_external.c:134-170) -> SoA Q[f][c]
__global__ void aos_to_soa_kernel(const double *__restrict__ aos, double *__restrict__ soa,
                                  long long ncells, long long stride)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        const double2 a = reinterpret_cast<const double2 *>(aos)[2 * c];
        const double2 b = reinterpret_cast<const double2 *>(aos)[2 * c + 1];
        soa[c] = a.x;
        soa[stride + c] = a.y;
        soa[2 * stride + c] = b.x;
        soa[3 * stride + c] = b.y;
    }
}

__global__ void soa_to_aos_kernel(const double *__restrict__ soa, double *__restrict__ aos,
                                  long long ncells, long long stride)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        double2 a, b;
        a.x = soa[c];
        a.y = soa[stride + c];
        b.x = soa[2 * stride + c];
        b.y = soa[3 * stride + c];
        reinterpret_cast<double2 *>(aos)[2 * c] = a;
        reinterpret_cast<double2 *>(aos)[2 * c + 1] = b;
    }
}

// sum over cells of volume * Q_f, per block partials in block order
template <int N>
__global__ void __launch_bounds__(256) totals_kernel(const QuadDesc *quads, const double *q,
                                                     long long stride, int nquad, double *partials)
{
    constexpr int NN = N * N;
    __shared__ double red[4][8];
    const double s = 2.0 / (double)N;
    double acc[4] = {0, 0, 0, 0};
    const long long ncells = (long long)nquad * NN;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells;
         c += (long long)gridDim.x * blockDim.x) {
        int qd = (int)(c / NN);
        int r = (int)(c - (long long)qd * NN);
        int i = r % N, j = r / N;
        const double *g = quads[qd].corner;
        double x1, y1, x2, y2, x3, y3, x4, y4;
        bilinear_node(g, s * i - 1.0, s * j - 1.0, x1, y1);
        bilinear_node(g, s * (i + 1) - 1.0, s * j - 1.0, x2, y2);
        bilinear_node(g, s * i - 1.0, s * (j + 1) - 1.0, x3, y3);
        bilinear_node(g, s * (i + 1) - 1.0, s * (j + 1) - 1.0, x4, y4);
        double vol = subcell_volume(x1, y1, x2, y2, x3, y3, x4, y4);
#pragma unroll
        for (int f = 0; f < 4; ++f) acc[f] += vol * q[f * stride + c];
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        double v = warp_sum(acc[f]);
        if ((threadIdx.x & 31) == 0) red[f][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
        partials[4 * blockIdx.x + threadIdx.x] = t;
    }
}

__device__ __forceinline__ double rel_jump(double a, double b) { return fabs(a - b) / fmin(a, b); }

// Plain indicator of solver_tag_feature.F90:9-52 (methods 1: any rho <= tol,
// 2: any rho >= tol; 3 and 4 are empty in the reference) plus method 5
// (extension): largest relative density jump >= tol between adjacent cells
// of the patch, or between an edge cell and the neighbour cell(s) it
// exchanges a face flux with (the flux kernels' index pairing, hanging
// faces included). One warp per quad.
template <int N>
__global__ void tag_kernel(const double *rho, const QuadDesc *quads, int nquad, int nmeth, TagMethods m,
                           int *tags)
{
    constexpr int NN = N * N;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nquad) return;
    const double *p = rho + (long long)warp * NN;
    int tag = 0;
    for (int k = 0; k < nmeth; ++k) {
        int hit = 0;
        double tol = m.tol[k];
        for (int c = lane; c < NN; c += 32) {
            double r = p[c];
            if (m.method[k] == 1 && r <= tol) hit = 1;
            if (m.method[k] == 2 && r >= tol) hit = 1;
            if (m.method[k] == 5) {
                int i = c % N, j = c / N;
                double jump = 0.0;
                if (i + 1 < N) jump = fmax(jump, rel_jump(p[c + 1], r));
                if (j + 1 < N) jump = fmax(jump, rel_jump(p[c + N], r));
                if (jump >= tol) hit = 1;
            }
        }
        if (m.method[k] == 5) {
            for (int e = lane; e < 4 * N; e += 32) {
                const int s = e / N, mm = e % N;
                const SideDesc &d = quads[warp].side[s];
                const int own = (s == 0) ? mm * N : (s == 1) ? mm * N + N - 1 : (s == 2) ? mm : (N - 1) * N + mm;
                const int fc = facing_cell<N>(s, mm);
                if (d.kind == kSideFull || d.kind == kSideFineHang || d.kind == kSideCoarseHang) {
                    if (rel_jump(p[own], rho[(long long)d.nbr0 * NN + fc]) >= tol) hit = 1;
                }
                if (d.kind == kSideCoarseHang) {
                    if (rel_jump(p[own], rho[(long long)d.nbr1 * NN + fc]) >= tol) hit = 1;
                }
            }
        }
        if (__any_sync(0xffffffffu, hit)) tag = 1;
    }
    if (lane == 0) tags[warp] = tag;
}

// refine = inject the parent patch into a child (solver_refine_operator_2d.F90:49-52),
// coarsen = (uc1+uc2+uc3+uc4)*0.25 (solver_coarsen_operator_2d.F90:49-50).
template <int N>
__global__ void remap_kernel(const double *__restrict__ qold, long long stride_old,
                             double *__restrict__ qnew, long long stride_new, const int *kind,
                             const int *src, int nquad_new)
{
    constexpr int NN = N * N;
    const long long total = (long long)nquad_new * NN;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        int q = (int)(c / NN);
        int r = (int)(c - (long long)q * NN);
        int s = src[q];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            double v;
            if (kind[q] == 0) {
                v = qold[f * stride_old + (long long)s * NN + r];
            } else {
                double u1 = qold[f * stride_old + (long long)s * NN + r];
                double u2 = qold[f * stride_old + (long long)(s + 1) * NN + r];
                double u3 = qold[f * stride_old + (long long)(s + 2) * NN + r];
                double u4 = qold[f * stride_old + (long long)(s + 3) * NN + r];
                double sum = u1 + u2 + u3 + u4;
                v = 0.25 * sum;
            }
            qnew[f * stride_new + c] = v;
        }
    }
}

// Re-arms the step slots after an in-place mesh change without a host
// round trip: the current step's start time is kept, every slot takes the
// dt cap, and the per-segment counters restart (the device form of the
// host-side priming that follows an upload).
__global__ void rearm_kernel(DeviceScalars *s, int slot_now, double cap)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double t = s->slot[slot_now].time;
    const unsigned long long bits = (unsigned long long)__double_as_longlong(cap);
    for (int k = 0; k < 3; ++k) {
        s->slot[k].dt_bits = bits;
        s->slot[k].time = t;
    }
    s->norm_sq = 0.0;
    s->dt_used = 0.0;
    s->done_blocks = 0u;
    s->flags = 0;
    s->steps = 0;
    s->work_next = 0u;
}

static int grid_for(long long work, int block)
{
    long long g = (work + block - 1) / block;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    return int(g);
}

cudaError_t launch_aos_to_soa(const double *aos, double *soa, long long ncells, long long stride,
                              cudaStream_t st)
{
    aos_to_soa_kernel<<<grid_for(ncells, 256), 256, 0, st>>>(aos, soa, ncells, stride);
    return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(const double *soa, double *aos, long long ncells, long long stride,
                              cudaStream_t st)
{
    soa_to_aos_kernel<<<grid_for(ncells, 256), 256, 0, st>>>(soa, aos, ncells, stride);
    return cudaGetLastError();
}

int totals_grid(long long ncells) { return grid_for(ncells, 256); }

cudaError_t launch_totals(int n, const QuadDesc *quads, const double *q, long long stride, int nquad,
                          double *partials, int grid, cudaStream_t st)
{
    switch (n) {
    case 2: totals_kernel<2><<<grid, 256, 0, st>>>(quads, q, stride, nquad, partials); break;
    case 4: totals_kernel<4><<<grid, 256, 0, st>>>(quads, q, stride, nquad, partials); break;
    case 8: totals_kernel<8><<<grid, 256, 0, st>>>(quads, q, stride, nquad, partials); break;
    case 16: totals_kernel<16><<<grid, 256, 0, st>>>(quads, q, stride, nquad, partials); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_tag(int n, const double *rho, const QuadDesc *quads, int nquad, int nmeth,
                       const TagMethods &m, int *tags, cudaStream_t st)
{
    int blocks = (nquad * 32 + 255) / 256;
    if (blocks < 1) blocks = 1;
    switch (n) {
    case 2: tag_kernel<2><<<blocks, 256, 0, st>>>(rho, quads, nquad, nmeth, m, tags); break;
    case 4: tag_kernel<4><<<blocks, 256, 0, st>>>(rho, quads, nquad, nmeth, m, tags); break;
    case 8: tag_kernel<8><<<blocks, 256, 0, st>>>(rho, quads, nquad, nmeth, m, tags); break;
    case 16: tag_kernel<16><<<blocks, 256, 0, st>>>(rho, quads, nquad, nmeth, m, tags); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_rearm(DeviceScalars *scal, int slot_now, double cap, cudaStream_t st)
{
    rearm_kernel<<<1, 32, 0, st>>>(scal, slot_now, cap);
    return cudaGetLastError();
}

cudaError_t launch_remap(int n, const double *qold, long long stride_old, double *qnew,
                         long long stride_new, const int *kind, const int *src, int nquad_new,
                         cudaStream_t st)
{
    long long work = (long long)nquad_new * n * n;
    int g = grid_for(work, 256);
    switch (n) {
    case 2: remap_kernel<2><<<g, 256, 0, st>>>(qold, stride_old, qnew, stride_new, kind, src, nquad_new); break;
    case 4: remap_kernel<4><<<g, 256, 0, st>>>(qold, stride_old, qnew, stride_new, kind, src, nquad_new); break;
    case 8: remap_kernel<8><<<g, 256, 0, st>>>(qold, stride_old, qnew, stride_new, kind, src, nquad_new); break;
    case 16: remap_kernel<16><<<g, 256, 0, st>>>(qold, stride_old, qnew, stride_new, kind, src, nquad_new); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace amrgpu
