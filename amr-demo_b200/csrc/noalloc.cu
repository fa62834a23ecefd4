// noalloc.cu -- conservation totals of a device-resident state without any
// device or host allocation.
//
// Some callers cannot let a library allocate: an AMR driver that hands all
// device memory to its own pool at start-up (a cudaMalloc from here would
// fail or fragment that pool), or one that checks conservation inside its
// time-step loop on a busy device, where cudaFree's implicit device-wide
// synchronisation would stall every other stream. This entry point keeps
// its scratch in a fixed-size array in the library's device image instead.
//
// The scratch holds one partial sum per quad, so the result is summed in
// quad order and does not depend on the launch shape. Its size bounds the
// number of quads a call accepts (AMRGPU_NOALLOC_MAX_QUADS); larger requests
// are rejected before any GPU work. Every GPU that loads the library holds
// the array until the process exits. All calls share it and it keeps the
// last call's contents; calls that overlap on the GPU (different streams,
// or different host threads on one device) race on it.
#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "amrgpu_internal.h"
#include "stage_kernel.cuh"

namespace amrgpu {

static __device__ __align__(256) double g_totals_scratch[(AMRGPU_NOALLOC_MAX_QUADS + 1) * 4];

// device address of g_totals_scratch per device, found once per device;
// atomic so that two host threads making their first call on one device at
// the same time both publish (the same) address without a data race
static std::atomic<double *> g_scratch_addr[64];

// one block per quad group: sum of vol * Q_f over each quad's cells, in
// cell order, written to the quad's own scratch slot
template <int N>
__global__ void __launch_bounds__(128) quad_totals_kernel(const double *q, long long stride,
                                                          const double *corners, int nquad,
                                                          double *scratch)
{
    constexpr int NN = N * N;
    const int qd = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (qd >= nquad) return;
    const double *g = corners + 8 * (long long)qd;
    const double s = 2.0 / (double)N;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = lane; c < NN; c += 32) {
        int i = c % N, j = c / N;
        double x1, y1, x2, y2, x3, y3, x4, y4;
        bilinear_node(g, s * i - 1.0, s * j - 1.0, x1, y1);
        bilinear_node(g, s * (i + 1) - 1.0, s * j - 1.0, x2, y2);
        bilinear_node(g, s * i - 1.0, s * (j + 1) - 1.0, x3, y3);
        bilinear_node(g, s * (i + 1) - 1.0, s * (j + 1) - 1.0, x4, y4);
        double vol = subcell_volume(x1, y1, x2, y2, x3, y3, x4, y4);
        long long gi = (long long)qd * NN + c;
#pragma unroll
        for (int f = 0; f < 4; ++f) acc[f] += vol * q[f * stride + gi];
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        double v = warp_sum(acc[f]);
        if (lane == 0) scratch[4 * (long long)qd + f] = v;
    }
}

// sums the per-quad partials in quad order into the scratch tail
__global__ void __launch_bounds__(128) totals_finish_kernel(double *scratch, int nquad)
{
    const int f = threadIdx.x;
    if (f >= 4) return;
    double t = 0.0;
    for (int q = 0; q < nquad; ++q) t += scratch[4 * (long long)q + f];
    scratch[4 * (long long)AMRGPU_NOALLOC_MAX_QUADS + f] = t;
}

}  // namespace amrgpu

using namespace amrgpu;

extern "C" int amrgpu_totals_noalloc(const double *q_device, long long field_stride, const double *corners_device,
                                     int nquad, int n, double totals[4], void *stream)
{
    if (!q_device || !corners_device || !totals || nquad < 0 || field_stride < (long long)nquad * n * n) {
        set_error(AMRGPU_ERR_ARG, "totals_noalloc: null pointer or inconsistent sizes");
        return AMRGPU_ERR_ARG;
    }
    if (nquad > AMRGPU_NOALLOC_MAX_QUADS) {
        set_error(AMRGPU_ERR_TOO_LARGE, "totals_noalloc: " + std::to_string(nquad) + " quads exceed the " +
                                            std::to_string(AMRGPU_NOALLOC_MAX_QUADS) +
                                            "-quad scratch array; use amrgpu_session_totals");
        return AMRGPU_ERR_TOO_LARGE;
    }
    if (n != 2 && n != 4 && n != 8 && n != 16) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "totals_noalloc: patch size must be 2, 4, 8 or 16");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(AMRGPU_ERR_CUDA, std::string("totals_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return AMRGPU_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "totals_noalloc: device index " + std::to_string(dev) +
                                              " is outside the 64 devices this entry point tracks");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    // set-up, once per device, with that device current: the host-side name
    // g_totals_scratch is only a stand-in, the kernels need the device address
    double *scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_totals_scratch);
        if (e != cudaSuccess || !p) {
            set_error(AMRGPU_ERR_CUDA, std::string("totals_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return AMRGPU_ERR_CUDA;
        }
        scratch = static_cast<double *>(p);
        g_scratch_addr[dev].store(scratch, std::memory_order_release);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (nquad > 0) {
        const int per_block = 4;  // warps (quads) per 128-thread block
        dim3 grid((nquad + per_block - 1) / per_block);
        switch (n) {
        case 2: quad_totals_kernel<2><<<grid, 128, 0, st>>>(q_device, field_stride, corners_device, nquad, scratch); break;
        case 4: quad_totals_kernel<4><<<grid, 128, 0, st>>>(q_device, field_stride, corners_device, nquad, scratch); break;
        case 8: quad_totals_kernel<8><<<grid, 128, 0, st>>>(q_device, field_stride, corners_device, nquad, scratch); break;
        default: quad_totals_kernel<16><<<grid, 128, 0, st>>>(q_device, field_stride, corners_device, nquad, scratch); break;
        }
    }
    totals_finish_kernel<<<1, 32, 0, st>>>(scratch, nquad);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(totals, scratch + 4 * (long long)AMRGPU_NOALLOC_MAX_QUADS, 4 * sizeof(double),
                            cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_error(AMRGPU_ERR_CUDA, std::string("totals_noalloc: ") + cudaGetErrorString(e));
        return AMRGPU_ERR_CUDA;
    }
    return AMRGPU_OK;
}
