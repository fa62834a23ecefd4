// mixed.cu -- kernels around the row sweep for meshes that mix 8x8 and
// 16x16 patches (extension: the reference fixes one patch size at compile
// time, src/amr/src/var_defines.h:29-32). Every quad's state starts at its
// MixDesc::base cell; these kernels take the per-quad size from MixDesc
// instead of a template parameter:
//   cfl_mixed_kernel     the FP32-flux form's CFL step of a state (segment
//                        prologue), the stage kernel's candidate per cell
//   totals_mixed_kernel  conservation totals sum(vol * Q_f)
//   tag_mixed_kernel     the plain indicator (methods 1, 2, 5), the jump
//                        across an edge taken with the cell the flux kernel
//                        pairs (geometric position for unequal sizes)
//   remap_mixed_kernel   refine / coarsen / copy of a regrid, with a size
//                        change resampled by position
//   build_mix (3 kernels + 2 scans)  the descriptors and work list of a
//                        forest regridded on the device, sizes by level
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "device_common.cuh"
#include "flux_fp32.cuh"
#include "misc_kernels.h"
#include "stage_kernel.cuh"

namespace amrgpu {

// One warp per quad (grid-stride over quads); the block's minimum goes to
// the slot by one 64-bit atomicMin on the order-preserving image, as the
// uniform prologue does. Same candidate and rectangle volume as the stage
// kernel's last stage, so a step's dt does not depend on where a segment
// starts.
__global__ void __launch_bounds__(256) cfl_mixed_kernel(const CflArgs a)
{
    __shared__ double red[8];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double best = __longlong_as_double((long long)a.scal->slot[a.slot].dt_bits);
    for (int q = warp; q < a.nquad; q += nwarps) {
        const MixDesc md = a.mix[q];
        const double *g = a.quads[q].corner;
        const double hx = (g[2] - g[0]) / (double)md.n, hy = (g[5] - g[1]) / (double)md.n;
        for (int c = lane; c < md.n * md.n; c += 32) {
            double q4[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) q4[f] = a.qin[f * a.stride + md.base + c];
            const double cand = cfl_candidate_fp32(q4, hx * hy, a.cfl);
            if (cand < best) best = cand;
        }
    }
    best = warp_min(best);
    if (lane == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = (red[w] < best) ? red[w] : best;
        atomicMin(&a.scal->slot[a.slot].dt_bits, (unsigned long long)__double_as_longlong(best));
    }
}

// sum over cells of volume * Q_f (volume from the bilinear sub-cell nodes,
// as the uniform totals kernel), one warp per quad, block partials in
// block order.
__global__ void __launch_bounds__(256) totals_mixed_kernel(const QuadDesc *quads, const MixDesc *mix,
                                                           const double *q, long long stride, int nquad,
                                                           double *partials)
{
    __shared__ double red[4][8];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double acc[4] = {0, 0, 0, 0};
    for (int qd = warp; qd < nquad; qd += nwarps) {
        const int n = mix[qd].n;
        const long long base = mix[qd].base;
        const double s = 2.0 / (double)n;
        const double *g = quads[qd].corner;
        for (int r = lane; r < n * n; r += 32) {
            const int i = r % n, j = r / n;
            double x1, y1, x2, y2, x3, y3, x4, y4;
            bilinear_node(g, s * i - 1.0, s * j - 1.0, x1, y1);
            bilinear_node(g, s * (i + 1) - 1.0, s * j - 1.0, x2, y2);
            bilinear_node(g, s * i - 1.0, s * (j + 1) - 1.0, x3, y3);
            bilinear_node(g, s * (i + 1) - 1.0, s * (j + 1) - 1.0, x4, y4);
            const double vol = subcell_volume(x1, y1, x2, y2, x3, y3, x4, y4);
#pragma unroll
            for (int f = 0; f < 4; ++f) acc[f] += vol * q[f * stride + base + r];
        }
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        double v = warp_sum(acc[f]);
        if (lane == 0) red[f][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
        partials[4 * blockIdx.x + threadIdx.x] = t;
    }
}

__device__ __forceinline__ double rel_jump_m(double a, double b) { return fabs(a - b) / fmin(a, b); }

// Position of own edge cell m on side s of a quad of size n in its
// neighbour's edge (size nn): the first neighbour cell the flux kernel pairs
// with it (geometric for unequal sizes, the same index otherwise) and which
// of a coarse edge's two fine neighbours holds it.
__device__ __forceinline__ void edge_partner(const SideDesc &d, const MixSide &ms, int n, int m, int &p,
                                             int &which)
{
    const int nn = ms.n;
    which = 0;
    p = m;
    if (nn == n) return;
    if (d.kind == kSideFull) {
        p = nn > n ? m * (nn / n) : m * nn / n;
    } else if (d.kind == kSideCoarseHang) {
        const int g = 2 * nn >= n ? m * (2 * nn / n) : m * 2 * nn / n;
        which = (g / nn) ^ ms.half;
        p = g % nn;
    } else {
        p = (ms.half * n + m) * nn / (2 * n);
    }
}

__device__ __forceinline__ int facing_rt(int s, int p, int n)
{
    if (s == 0) return p * n + (n - 1);
    if (s == 1) return p * n;
    if (s == 2) return (n - 1) * n + p;
    return p;
}

// The plain indicator of tag_kernel (solver_tag_feature.F90:9-52 methods 1
// and 2, and the relative density jump of method 5) on a mixed mesh. One
// warp per quad.
__global__ void tag_mixed_kernel(const double *rho, const QuadDesc *quads, const MixDesc *mix, int nquad,
                                 int nmeth, TagMethods m, int *tags)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nquad) return;
    const MixDesc md = mix[warp];
    const int N = md.n, NN = N * N;
    const double *p = rho + md.base;
    int tag = 0;
    for (int k = 0; k < nmeth; ++k) {
        int hit = 0;
        const double tol = m.tol[k];
        for (int c = lane; c < NN; c += 32) {
            const double r = p[c];
            if (m.method[k] == 1 && r <= tol) hit = 1;
            if (m.method[k] == 2 && r >= tol) hit = 1;
            if (m.method[k] == 5) {
                const int i = c % N, j = c / N;
                double jump = 0.0;
                if (i + 1 < N) jump = fmax(jump, rel_jump_m(p[c + 1], r));
                if (j + 1 < N) jump = fmax(jump, rel_jump_m(p[c + N], r));
                if (jump >= tol) hit = 1;
            }
        }
        if (m.method[k] == 5) {
            for (int e = lane; e < 4 * N; e += 32) {
                const int s = e / N, mm = e % N;
                const SideDesc &d = quads[warp].side[s];
                if (d.kind != kSideFull && d.kind != kSideFineHang && d.kind != kSideCoarseHang) continue;
                const MixSide &ms = md.side[s];
                const int own = (s == 0) ? mm * N : (s == 1) ? mm * N + N - 1 : (s == 2) ? mm : (N - 1) * N + mm;
                int pos, which;
                edge_partner(d, ms, N, mm, pos, which);
                const int fc = facing_rt(s, pos, ms.n);
                if (ms.n == N) {
                    if (rel_jump_m(p[own], rho[(long long)ms.base0 + fc]) >= tol) hit = 1;
                    if (d.kind == kSideCoarseHang && rel_jump_m(p[own], rho[(long long)ms.base1 + fc]) >= tol)
                        hit = 1;
                } else {
                    const long long nb = which ? ms.base1 : ms.base0;
                    if (rel_jump_m(p[own], rho[nb + fc]) >= tol) hit = 1;
                }
            }
        }
        if (__any_sync(0xffffffffu, hit)) tag = 1;
    }
    if (lane == 0) tags[warp] = tag;
}

// Value of cell (i, j) of a patch of size n read from a source patch of size
// ns at src (field stride stride): the same cell when the sizes agree, the
// covering cell when the new patch is finer (ns = n/2), the mean of the four
// covered cells, summed in row order, when it is coarser (ns = 2n).
__device__ __forceinline__ double resample(const double *src, int ns, int n, int i, int j)
{
    if (ns == n) return src[j * n + i];
    if (ns * 2 == n) return src[(j / 2) * ns + (i / 2)];
    const double a = src[(2 * j) * ns + 2 * i], b = src[(2 * j) * ns + 2 * i + 1];
    const double c = src[(2 * j + 1) * ns + 2 * i], d = src[(2 * j + 1) * ns + 2 * i + 1];
    return 0.25 * (((a + b) + c) + d);
}

// The regrid remap on a mixed mesh: kind 0 copies (or, for a refined child,
// injects) source quad src[q]; kind 1 averages the four children src[q] ..
// src[q]+3 cell by cell (the reference's operators,
// solver_refine_operator_2d.F90:49-52, solver_coarsen_operator_2d.F90:49-50);
// a patch-size change between source and target is resampled by position
// (resample above). Same-size remaps give the uniform kernel's bits. One
// warp per new quad.
__global__ void remap_mixed_kernel(const double *__restrict__ qold, long long stride_old, const MixDesc *mold,
                                   double *__restrict__ qnew, long long stride_new, const MixDesc *mnew,
                                   const int *kind, const int *src, int nquad_new)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nquad_new) return;
    const int n = mnew[warp].n;
    const long long nb = mnew[warp].base;
    const int s = src[warp];
    const int ns = mold[s].n;
    for (int r = lane; r < n * n; r += 32) {
        const int i = r % n, j = r / n;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            double v;
            if (kind[warp] == 0) {
                v = resample(qold + f * stride_old + mold[s].base, ns, n, i, j);
            } else if (ns == n) {
                const double u1 = qold[f * stride_old + mold[s].base + r];
                const double u2 = qold[f * stride_old + mold[s + 1].base + r];
                const double u3 = qold[f * stride_old + mold[s + 2].base + r];
                const double u4 = qold[f * stride_old + mold[s + 3].base + r];
                const double sum = u1 + u2 + u3 + u4;
                v = 0.25 * sum;
            } else {
                // average of the children at each source position, then
                // resampled to the new size
                auto child_mean = [&](int ci, int cj) {
                    const int rr = cj * ns + ci;
                    const double u1 = qold[f * stride_old + mold[s].base + rr];
                    const double u2 = qold[f * stride_old + mold[s + 1].base + rr];
                    const double u3 = qold[f * stride_old + mold[s + 2].base + rr];
                    const double u4 = qold[f * stride_old + mold[s + 3].base + rr];
                    const double sum = u1 + u2 + u3 + u4;
                    return 0.25 * sum;
                };
                if (ns * 2 == n) {
                    v = child_mean(i / 2, j / 2);
                } else {
                    const double a = child_mean(2 * i, 2 * j), b = child_mean(2 * i + 1, 2 * j);
                    const double c = child_mean(2 * i, 2 * j + 1), d = child_mean(2 * i + 1, 2 * j + 1);
                    v = 0.25 * (((a + b) + c) + d);
                }
            }
            qnew[f * stride_new + nb + r] = v;
        }
    }
}

// ---- descriptors of a mixed mesh built on the device (the forest's
// leaves and the new quad descriptors already there; sizes by level)

__global__ void mix_sizes_kernel(const int4 *leaves, int nq, SizeRule rule, int *cells, int *flag16)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q > nq) return;
    if (q == nq) {  // the scans' closing element
        cells[q] = 0;
        flag16[q] = 0;
        return;
    }
    const int n = rule.size[leaves[q].y & 31];
    cells[q] = n * n;
    flag16[q] = n == 16 ? 1 : 0;
}

__global__ void mix_desc_kernel(const int4 *leaves, const QuadDesc *quads, int nq, SizeRule rule, const int *base,
                                const int *pos16, MixDesc *out, int *work, int *status)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q == 0) {
        status[1] = base[nq];   // cells
        status[2] = pos16[nq];  // 16x16 quads
    }
    if (q >= nq) return;
    const int n = rule.size[leaves[q].y & 31];
    MixDesc md;
    md.n = n;
    md.base = base[q];
    md.level = leaves[q].y;
    md.pad = 0;
    const QuadDesc &qd = quads[q];
    for (int k = 0; k < 4; ++k) {
        const SideDesc &d = qd.side[k];
        MixSide ms{n, 0, 0, 0};
        auto along = [&](int p) { return quads[p].corner[k < 2 ? 1 : 0]; };
        if (d.kind == kSideFull || d.kind == kSideCoarseHang || d.kind == kSideFineHang) {
            ms.n = rule.size[leaves[d.nbr0].y & 31];
            ms.base0 = base[d.nbr0];
        }
        if (d.kind == kSideCoarseHang) {
            if (rule.size[leaves[d.nbr1].y & 31] != ms.n) atomicOr(&status[0], 1);
            ms.base1 = base[d.nbr1];
            ms.half = along(d.nbr1) < along(d.nbr0) ? 1 : 0;
        } else if (d.kind == kSideFineHang) {
            const double *g = qd.corner;
            const double len = k < 2 ? fabs(g[5] - g[1]) : fabs(g[2] - g[0]);
            ms.half = along(q) - along(d.nbr0) > 0.25 * len ? 1 : 0;
        }
        md.side[k] = ms;
    }
    out[q] = md;
    const int c16 = pos16[nq];
    work[n == 16 ? pos16[q] : c16 + (q - pos16[q])] = q;
}

size_t build_mix_scan_bytes(int nq)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int *)nullptr, (int *)nullptr, (nq > 0 ? nq : 1) + 1);
    return bytes;
}

cudaError_t launch_build_mix(const int4 *leaves, const QuadDesc *quads, int nq, const SizeRule &rule, MixDesc *out,
                             int *work, int *cells, int *flag16, int *base, int *pos16, void *scan_tmp,
                             size_t scan_bytes, int *status, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(status, 0, 3 * sizeof(int), st);
    if (e != cudaSuccess) return e;
    const int g = (nq + 1 + 255) / 256;
    mix_sizes_kernel<<<g, 256, 0, st>>>(leaves, nq, rule, cells, flag16);
    e = cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, cells, base, nq + 1, st);
    if (e != cudaSuccess) return e;
    e = cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, flag16, pos16, nq + 1, st);
    if (e != cudaSuccess) return e;
    mix_desc_kernel<<<(std::max(nq, 1) + 255) / 256, 256, 0, st>>>(leaves, quads, nq, rule, base, pos16, out, work,
                                                                   status);
    return cudaGetLastError();
}

static int warps_grid(int nquad)
{
    long long g = ((long long)nquad * 32 + 255) / 256;
    if (g < 1) g = 1;
    return int(g);
}

const void *cfl_kernel_mixed() { return (const void *)cfl_mixed_kernel; }

int totals_mixed_grid(int nquad)
{
    int g = warps_grid(nquad);
    return g > 148 * 8 ? 148 * 8 : g;
}

cudaError_t launch_totals_mixed(const QuadDesc *quads, const MixDesc *mix, const double *q, long long stride,
                                int nquad, double *partials, int grid, cudaStream_t st)
{
    totals_mixed_kernel<<<grid, 256, 0, st>>>(quads, mix, q, stride, nquad, partials);
    return cudaGetLastError();
}

cudaError_t launch_tag_mixed(const double *rho, const QuadDesc *quads, const MixDesc *mix, int nquad, int nmeth,
                             const TagMethods &m, int *tags, cudaStream_t st)
{
    tag_mixed_kernel<<<warps_grid(nquad), 256, 0, st>>>(rho, quads, mix, nquad, nmeth, m, tags);
    return cudaGetLastError();
}

cudaError_t launch_remap_mixed(const double *qold, long long stride_old, const MixDesc *mold, double *qnew,
                               long long stride_new, const MixDesc *mnew, const int *kind, const int *src,
                               int nquad_new, cudaStream_t st)
{
    remap_mixed_kernel<<<warps_grid(nquad_new), 256, 0, st>>>(qold, stride_old, mold, qnew, stride_new, mnew, kind,
                                                              src, nquad_new);
    return cudaGetLastError();
}

}  // namespace amrgpu
