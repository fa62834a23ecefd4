// halo.cu -- ghost-quad exchange kernels of a sharded mesh.
//
// A rank's mesh holds its ncell local quads followed by its ghost quads
// (copies of neighbours owned by other ranks), grouped by owning rank in
// ascending order, as physics_mpi.c:54 lays out the reference's ghosts
// ("ghosts are always at the end and stacked in order of processor"). Before
// every RK stage the ghost patches of the stage's input buffer are refreshed
// from their owners (rk_time_integrators.c:227,243,259 call
// physics_mpi_real_to_ghost before each physics_rhs).
//
// Wire format of one quad: its 4 fields, each the n*n cells of the patch in
// the SoA order the state uses -- 4*n*n doubles. pack gathers a list of
// local quads into consecutive records (the reference's send buffer,
// physics_mpi.c:80-91); unpack writes consecutive records into ghost slots
// ncell .. ncell+count-1 (the reference's receives straight into the ghost
// storage, physics_mpi.c:60-77). Both move 2 doubles per thread; n*n is even
// for every supported patch size.
//
// Edge-strip format (pack_edges / unpack_edges): the stage kernels read a
// ghost quad only at the cells that face their own quads -- its one-cell
// edge rows and columns -- so a ghost can travel as its four edge strips:
// per field the n cells of side 0 (column 0), side 1 (column n-1), side 2
// (row 0), side 3 (row n-1), 16*n doubles (corner cells twice), 4x fewer
// than the whole patch at 16x16, 2x at 8x8. A ghost's interior cells are
// left as they were; nothing reads them.
#include <cuda_runtime.h>

#include "halo_kernels.h"

namespace amrgpu {

__global__ void halo_pack_kernel(const double *__restrict__ q, long long stride, int nn,
                                 const int *__restrict__ list, int count, double *__restrict__ out)
{
    const int half = nn >> 1;                       // double2 per field of a quad
    const long long total = (long long)count * 4 * half;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / (4 * half));
        const int r = (int)(e - (long long)k * 4 * half);
        const int f = r / half, c2 = r - f * half;
        const long long src = (long long)f * stride + (long long)__ldg(list + k) * nn + 2 * c2;
        const double2 v = *reinterpret_cast<const double2 *>(q + src);
        reinterpret_cast<double2 *>(out)[e] = v;
    }
}

__global__ void halo_unpack_kernel(double *__restrict__ q, long long stride, int nn, int first_quad,
                                   int count, const double *__restrict__ in)
{
    const int half = nn >> 1;
    const long long total = (long long)count * 4 * half;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / (4 * half));
        const int r = (int)(e - (long long)k * 4 * half);
        const int f = r / half, c2 = r - f * half;
        const long long dst = (long long)f * stride + (long long)(first_quad + k) * nn + 2 * c2;
        *reinterpret_cast<double2 *>(q + dst) = reinterpret_cast<const double2 *>(in)[e];
    }
}

// Cell of a patch of size n at position p of side s's edge strip.
__device__ __forceinline__ int strip_cell(int s, int p, int n)
{
    if (s == 0) return p * n;
    if (s == 1) return p * n + n - 1;
    if (s == 2) return p;
    return (n - 1) * n + p;
}

__global__ void halo_pack_edges_kernel(const double *__restrict__ q, long long stride, int n,
                                       const int *__restrict__ list, int count, double *__restrict__ out)
{
    const int per = 16 * n;  // doubles per quad: 4 fields x 4 sides x n
    const long long total = (long long)count * per;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / per);
        const int r = (int)(e - (long long)k * per);
        const int f = r / (4 * n), s = (r / n) & 3, p = r % n;
        out[e] = q[(long long)f * stride + (long long)__ldg(list + k) * n * n + strip_cell(s, p, n)];
    }
}

__global__ void halo_unpack_edges_kernel(double *__restrict__ q, long long stride, int n, int first_quad,
                                         int count, const double *__restrict__ in)
{
    const int per = 16 * n;
    const long long total = (long long)count * per;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / per);
        const int r = (int)(e - (long long)k * per);
        const int f = r / (4 * n), s = (r / n) & 3, p = r % n;
        q[(long long)f * stride + (long long)(first_quad + k) * n * n + strip_cell(s, p, n)] = in[e];
    }
}

namespace {
int halo_grid(long long pairs, int sms)
{
    long long g = (pairs + 255) / 256;
    long long cap = (long long)sms * 8;
    if (g > cap) g = cap;
    return g < 1 ? 1 : int(g);
}
}  // namespace

cudaError_t launch_halo_pack(const double *q, long long stride, int n, const int *list, int count, double *out,
                             int sms, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    const int nn = n * n;
    halo_pack_kernel<<<halo_grid((long long)count * 2 * nn, sms), 256, 0, st>>>(q, stride, nn, list, count, out);
    return cudaGetLastError();
}

cudaError_t launch_halo_unpack(double *q, long long stride, int n, int first_quad, int count, const double *in,
                               int sms, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    const int nn = n * n;
    halo_unpack_kernel<<<halo_grid((long long)count * 2 * nn, sms), 256, 0, st>>>(q, stride, nn, first_quad,
                                                                                   count, in);
    return cudaGetLastError();
}

cudaError_t launch_halo_pack_edges(const double *q, long long stride, int n, const int *list, int count,
                                   double *out, int sms, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    halo_pack_edges_kernel<<<halo_grid((long long)count * 16 * n, sms), 256, 0, st>>>(q, stride, n, list, count,
                                                                                       out);
    return cudaGetLastError();
}

cudaError_t launch_halo_unpack_edges(double *q, long long stride, int n, int first_quad, int count,
                                     const double *in, int sms, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    halo_unpack_edges_kernel<<<halo_grid((long long)count * 16 * n, sms), 256, 0, st>>>(q, stride, n, first_quad,
                                                                                         count, in);
    return cudaGetLastError();
}

}  // namespace amrgpu
