// mlp.cu -- the learned refinement indicator: a 400-128-64-3 MLP with GELU
// that maps a patch's normalised conserved variables to coarsen / refine /
// keep, trained and evaluated on the GPU. Its weights are BF16, every GEMM
// accumulates in FP32 in tensor memory through tcgen05.mma (the only
// tensor-core use of the library), and the optimiser (AdamW) keeps FP32
// master weights. There is no counterpart in the reference: it stands in
// for the plain tagger (solver_tag_feature.F90:9-52 through
// hpc_amr_tag_feature, amr_external.h:92), which also labels its training
// data and judges it at run time.
//
// Data flow of one training step (batch B, rows = patches):
//   gather   X[B x 400], X^T[400 x B], y[B]        from the device dataset
//   fwd1     Z1 = X W1^T + b1,  H1 = gelu(Z1)      (also H1^T)
//   fwd2     Z2 = H1 W2^T + b2, H2 = gelu(Z2)      (also H2^T)
//   fwd3     L  = H2 W3^T + b3                     (3 logits, padded to 16)
//   loss     dL = softmax(L) - onehot(y)           (also dL^T), CE partials
//   bwd3     dZ2 = (dL W3) * gelu'(Z2)             (also dZ2^T)
//   bwd2     dZ1 = (dZ2 W2) * gelu'(Z1)^T          (transposed only)
//   wgrad    dW1 = dZ1^T X, dW2^T = H1^T dZ2, dW3^T = H2^T dL   (split over B)
//   bias     db = column sums of dZ1, dZ2, dL
//   adamw    FP32 master update, BF16 copies W and W^T refreshed
// Every GEMM is C[M x N] = A[M x K] B[N x K]^T with both operands K-major,
// which is why the forward and backward epilogues also write transposes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "amrgpu_internal.h"
#include "device_common.cuh"
#include "mlp_internal.h"
#include "stage_kernel.cuh"
#include "umma.cuh"

namespace amrgpu {

using bf16 = __nv_bfloat16;

enum Epi : int { kEpiHidden = 0, kEpiLogits = 1, kEpiBackHidden = 2, kEpiPartial = 3 };

struct GemmArgs {
    const bf16 *A;      // M x K, row stride lda (elements)
    long long lda;
    const bf16 *B;      // N x K, row stride ldb
    long long ldb;
    int M, N, K;        // N a multiple of 16, K of 8 (rows are read in 16-byte pieces)
    int k_per_split;    // K range of one blockIdx.z (multiple of 16)
    const float *bias;  // [N]                                (hidden, logits)
    float *zout;        // hidden: Z [M x N] or null; logits: [M x N]; partial: [splits][M x N]
    const float *zin;   // back-hidden: Z [M x N] for gelu'
    bf16 *hout;         // [M x N] row-major, or null
    bf16 *houtT;        // [N x ldt], or null
    long long ldt;
    int *err;           // error flags (bounded wait gave up)
};

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad_f(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

constexpr int kGemmKC = 64;  // K elements staged per chunk

template <int NT>
constexpr size_t gemm_smem_bytes()
{
    return size_t(128 + NT) * kGemmKC * 2 + 64;
}

// One CTA = 128 rows of C (one TMEM lane each) x NT columns, over the K
// range of its blockIdx.z. 4 warps: all stage operands, thread 0 issues the
// MMAs, every warp drains its 32 TMEM lanes in the epilogue.
template <int NT, int EPI>
__global__ void __launch_bounds__(128) mlp_gemm_kernel(const GemmArgs a)
{
    static_assert(NT % 16 == 0 && NT >= 16 && NT <= 256, "UMMA N for M = 128");
    constexpr int KC = kGemmKC;
    constexpr uint32_t NCOLS = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
    extern __shared__ __align__(128) unsigned char mlp_smem[];
    unsigned char *sA = mlp_smem;
    unsigned char *sB = mlp_smem + 128 * KC * 2;
    uint64_t *bar = reinterpret_cast<uint64_t *>(mlp_smem + (128 + NT) * KC * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * NT;
    const int kbeg = blockIdx.z * a.k_per_split;
    const int kend = min(a.K, kbeg + a.k_per_split);

    if (warp == 0) tmem_alloc(tslot, NCOLS);
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t idesc = umma_idesc_bf16_f32(128, NT);

    unsigned phase = 0;
    int ok = 1;
    for (int k0 = kbeg; k0 < kend && ok; k0 += KC) {
        const int kc = min(KC, kend - k0);
        for (int t = tid; t < 128 * (KC / 8); t += 128) {
            const int r = t / (KC / 8), c8 = t % (KC / 8);
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (m0 + r < a.M && c8 * 8 < kc)
                v = *reinterpret_cast<const uint4 *>(a.A + (long long)(m0 + r) * a.lda + k0 + c8 * 8);
            *reinterpret_cast<uint4 *>(sA + ((r >> 3) * (KC / 8) + c8) * 128 + (r & 7) * 16) = v;
        }
        for (int t = tid; t < NT * (KC / 8); t += 128) {
            const int r = t / (KC / 8), c8 = t % (KC / 8);
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (n0 + r < a.N && c8 * 8 < kc)
                v = *reinterpret_cast<const uint4 *>(a.B + (long long)(n0 + r) * a.ldb + k0 + c8 * 8);
            *reinterpret_cast<uint4 *>(sB + ((r >> 3) * (KC / 8) + c8) * 128 + (r & 7) * 16) = v;
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t abase = smem_u32(sA), bbase = smem_u32(sB);
            // a K range ending inside a 16-element step is zero-filled above
            for (int kk = 0; kk < (kc + 15) / 16; ++kk) {
                const uint64_t ad = umma_desc_kmajor(abase + kk * 256, 128, KC * 16);
                const uint64_t bd = umma_desc_kmajor(bbase + kk * 256, 128, KC * 16);
                umma_bf16_ss(tmem, ad, bd, idesc, (k0 > kbeg || kk > 0) ? 1u : 0u);
            }
            umma_commit(bar);
        }
        // the next chunk overwrites the operands only after these MMAs finish
        if (!mbar_wait_bounded(bar, phase, kWaitLimit)) ok = 0;
        phase ^= 1u;
        ok = __syncthreads_and(ok);
    }
    if (!ok) {
        // gave up waiting: report, let anything in flight finish (bounded),
        // release the tensor memory and leave without writing results
        if (tid == 0) atomicOr(a.err, kFlagTimeout);
        mbar_wait_bounded(bar, phase ^ 1u, kWaitLimit);
        tc_fence_before();
        __syncthreads();
        if (warp == 0) tmem_dealloc(tmem, NCOLS);
        return;
    }
    tc_fence_after();
    const bool any = kend > kbeg;
    const int row = m0 + warp * 32 + lane;
    const bool rv = row < a.M;
#pragma unroll 1
    for (int c0 = 0; c0 < NT; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        if (!any) {
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = 0.0f;
        }
        const int nb = n0 + c0;
        if (nb >= a.N) continue;
        if (EPI == kEpiHidden || EPI == kEpiLogits) {
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] += a.bias[nb + k];
            if (rv && a.zout) {
                float4 *dst = reinterpret_cast<float4 *>(a.zout + (long long)row * a.N + nb);
#pragma unroll
                for (int k = 0; k < 4; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
            }
            if (EPI == kEpiHidden) {
#pragma unroll
                for (int k = 0; k < 16; ++k) v[k] = gelu_f(v[k]);
            }
        } else if (EPI == kEpiBackHidden) {
            if (rv) {
                const float4 *zp = reinterpret_cast<const float4 *>(a.zin + (long long)row * a.N + nb);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float4 z = zp[k];
                    v[4 * k] *= gelu_grad_f(z.x);
                    v[4 * k + 1] *= gelu_grad_f(z.y);
                    v[4 * k + 2] *= gelu_grad_f(z.z);
                    v[4 * k + 3] *= gelu_grad_f(z.w);
                }
            }
        } else {  // kEpiPartial
            if (rv) {
                float4 *dst = reinterpret_cast<float4 *>(a.zout + ((long long)blockIdx.z * a.M + row) * a.N + nb);
#pragma unroll
                for (int k = 0; k < 4; ++k) dst[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
            }
            continue;
        }
        if (EPI == kEpiHidden || EPI == kEpiBackHidden) {
            if (rv && a.hout) {
                alignas(16) bf16 h[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) h[k] = __float2bfloat16_rn(v[k]);
                uint4 *dst = reinterpret_cast<uint4 *>(a.hout + (long long)row * a.N + nb);
                dst[0] = reinterpret_cast<const uint4 *>(h)[0];
                dst[1] = reinterpret_cast<const uint4 *>(h)[1];
            }
            if (rv && a.houtT) {
#pragma unroll
                for (int k = 0; k < 16; ++k) a.houtT[(long long)(nb + k) * a.ldt + row] = __float2bfloat16_rn(v[k]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, NCOLS);
}

template <int NT, int EPI>
static cudaError_t launch_gemm(const GemmArgs &a, int splits, cudaStream_t st)
{
    const void *k = (const void *)mlp_gemm_kernel<NT, EPI>;
    // cap residency at what tensor memory holds (512 columns per SM), so an
    // allocation never waits on a CTA that is not yet resident
    constexpr uint32_t ncols = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
    constexpr int per_sm = 512 / ncols;
    size_t smem = gemm_smem_bytes<NT>();
    const size_t cap = (size_t)220 * 1024 / per_sm + 1024;
    if (smem < cap) smem = cap;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.M + 127) / 128, (a.N + NT - 1) / NT, splits);
    void *args[] = {const_cast<GemmArgs *>(&a)};
    return cudaLaunchKernel(k, grid, dim3(128), args, smem, st);
}

// ---------------------------------------------------------------- features

// Patch features: the quad's n x n patch box-averaged to 8 x 8 (n = 8: as
// is, n = 16: 2 x 2 means) plus a one-cell ring from the neighbour cells
// its edge fluxes pair with (the flux kernels' index pairing; a coarse
// hanging side averages its two fine neighbours, a boundary side repeats
// the edge cells, the four ring corners repeat the patch corners), each
// field normalised by the patch's own mean state:
//   x0 = S (rho - mean rho) / mean rho
//   x1 = S (rho u - mean rho u) / (mean rho * a),   x2 likewise for rho v
//   x3 = S (rho E - mean rho E) / mean rho E
// with a the sound speed of the mean state and S = kFeatScale; layout
// X[q][c*100 + (J+1)*10 + (I+1)], I, J = -1..8.
template <int N>
__global__ void __launch_bounds__(128) features_kernel(const double *q, long long stride, const QuadDesc *quads,
                                                      int nquad, bf16 *X)
{
    constexpr int R = N / 8;
    constexpr int NN = N * N;
    __shared__ double P[4][10][10];
    __shared__ double red[4][4];
    const int quad = blockIdx.x;
    if (quad >= nquad) return;
    const int t = threadIdx.x;
    const double inv = 1.0 / (double)(R * R);
    if (t < 64) {
        const int I = t & 7, J = t >> 3;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            double s = 0.0;
#pragma unroll
            for (int dj = 0; dj < R; ++dj)
#pragma unroll
                for (int di = 0; di < R; ++di)
                    s += q[f * stride + (long long)quad * NN + (R * J + dj) * N + (R * I + di)];
            P[f][J + 1][I + 1] = s * inv;
        }
    } else if (t < 96) {
        const int sd = (t - 64) >> 3, M = (t - 64) & 7;
        const SideDesc d = quads[quad].side[sd];
        const double rinv = 1.0 / (double)R;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            double s = 0.0;
            for (int dm = 0; dm < R; ++dm) {
                const int m = R * M + dm;
                if (d.kind == kSideFull || d.kind == kSideFineHang) {
                    s += q[f * stride + (long long)d.nbr0 * NN + facing_cell<N>(sd, m)];
                } else if (d.kind == kSideCoarseHang) {
                    s += 0.5 * (q[f * stride + (long long)d.nbr0 * NN + facing_cell<N>(sd, m)] +
                                q[f * stride + (long long)d.nbr1 * NN + facing_cell<N>(sd, m)]);
                } else {
                    const int own = (sd == 0) ? m * N : (sd == 1) ? m * N + N - 1 : (sd == 2) ? m : (N - 1) * N + m;
                    s += q[f * stride + (long long)quad * NN + own];
                }
            }
            // box mean over the R cells facing this ring cell (own edge cells
            // for a boundary side are averaged across the edge only)
            const double v = s * rinv;
            if (sd == 0) P[f][M + 1][0] = v;
            else if (sd == 1) P[f][M + 1][9] = v;
            else if (sd == 2) P[f][0][M + 1] = v;
            else P[f][9][M + 1] = v;
        }
    }
    __syncthreads();
    if (t < 4) {
        const int cj = (t >> 1) ? 9 : 0, ci = (t & 1) ? 9 : 0;
        const int pj = (t >> 1) ? 8 : 1, pi = (t & 1) ? 8 : 1;
#pragma unroll
        for (int f = 0; f < 4; ++f) P[f][cj][ci] = P[f][pj][pi];
    }
    // means of the 8 x 8 patch, in a fixed order
    double m4[4] = {0.0, 0.0, 0.0, 0.0};
    if (t < 64) {
        const int I = t & 7, J = t >> 3;
#pragma unroll
        for (int f = 0; f < 4; ++f) m4[f] = P[f][J + 1][I + 1];
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) m4[f] = warp_sum(m4[f]);
    if ((t & 31) == 0 && t < 64) {
#pragma unroll
        for (int f = 0; f < 4; ++f) red[f][t >> 5] = m4[f];
    }
    __syncthreads();
    const double mr = (red[0][0] + red[0][1]) / 64.0;
    const double mu = (red[1][0] + red[1][1]) / 64.0;
    const double mv = (red[2][0] + red[2][1]) / 64.0;
    const double me = (red[3][0] + red[3][1]) / 64.0;
    const double pbar = 0.4 * (me - 0.5 * (mu * mu + mv * mv) / mr);
    const double c2 = 1.4 * pbar / mr;
    const double abar = sqrt(c2 > 1e-24 ? c2 : 1e-24);
    const double sc[4] = {kFeatScale / mr, kFeatScale / (mr * abar), kFeatScale / (mr * abar), kFeatScale / me};
    const double mm[4] = {mr, mu, mv, me};
    for (int k = t; k < kFeatIn; k += 128) {
        const int f = k / 100, r = k % 100;
        const double x = (P[f][r / 10][r % 10] - mm[f]) * sc[f];
        X[(long long)quad * kFeatIn + k] = __float2bfloat16_rn((float)x);
    }
}

// Largest relative density jump of a quad (the plain indicator's method 5
// quantity, as in tag_kernel): between adjacent cells of the patch and
// between an edge cell and the neighbour cell(s) its face flux pairs it
// with. Quads listed in `which` (or all when null), one warp each.
template <int N>
__global__ void jump_kernel(const double *rho, const QuadDesc *quads, const int *which, int count, double *jump)
{
    constexpr int NN = N * N;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= count) return;
    const int quad = which ? which[w] : w;
    const double *p = rho + (long long)quad * NN;
    auto rj = [](double x, double y) { return fabs(x - y) / fmin(x, y); };
    double J = 0.0;
    for (int c = lane; c < NN; c += 32) {
        const int i = c % N, j = c / N;
        if (i + 1 < N) J = fmax(J, rj(p[c + 1], p[c]));
        if (j + 1 < N) J = fmax(J, rj(p[c + N], p[c]));
    }
    for (int e = lane; e < 4 * N; e += 32) {
        const int s = e / N, mm = e % N;
        const SideDesc &d = quads[quad].side[s];
        const int own = (s == 0) ? mm * N : (s == 1) ? mm * N + N - 1 : (s == 2) ? mm : (N - 1) * N + mm;
        const int fc = facing_cell<N>(s, mm);
        if (d.kind == kSideFull || d.kind == kSideFineHang || d.kind == kSideCoarseHang)
            J = fmax(J, rj(p[own], rho[(long long)d.nbr0 * NN + fc]));
        if (d.kind == kSideCoarseHang) J = fmax(J, rj(p[own], rho[(long long)d.nbr1 * NN + fc]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) J = fmax(J, __shfl_xor_sync(0xffffffffu, J, o));
    if (lane == 0) jump[w] = J;
}

// ---------------------------------------------------------------- training kernels

// rows perm[b0 .. b0+B) of the dataset -> X[B x 400], X^T[400 x B], y[B]
__global__ void gather_kernel(const bf16 *Xall, const int *yall, const int *perm, int b0, int B, bf16 *X, bf16 *XT,
                              int *y)
{
    const int b = blockIdx.x;
    const int src = perm[b0 + b];
    for (int k = threadIdx.x; k < kFeatIn; k += blockDim.x) {
        const bf16 v = Xall[(long long)src * kFeatIn + k];
        X[(long long)b * kFeatIn + k] = v;
        XT[(long long)k * B + b] = v;
    }
    if (threadIdx.x == 0) y[b] = yall[src];
}

// Softmax cross-entropy on the first 3 of 16 logit columns:
// dL = softmax - onehot (not divided by B; the optimiser scales), written
// row-major and transposed (padding columns zero); per-block partial sums of
// the loss and of correct predictions.
__global__ void __launch_bounds__(256) softmax_ce_kernel(const float *L, const int *y, int B, bf16 *dL, bf16 *dLT,
                                                         double *loss_part, int *correct_part)
{
    __shared__ double sl[8];
    __shared__ int sc[8];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    double loss = 0.0;
    int corr = 0;
    if (b < B) {
        const float l0 = L[(long long)b * kOutPad], l1 = L[(long long)b * kOutPad + 1], l2 = L[(long long)b * kOutPad + 2];
        const float mx = fmaxf(l0, fmaxf(l1, l2));
        const float e0 = expf(l0 - mx), e1 = expf(l1 - mx), e2 = expf(l2 - mx);
        const float s = e0 + e1 + e2;
        const float p[3] = {e0 / s, e1 / s, e2 / s};
        const int yy = y[b];
        const float ly = yy == 0 ? l0 : yy == 1 ? l1 : l2;
        loss = (double)(mx + logf(s) - ly);
        const int arg = (l0 >= l1 && l0 >= l2) ? 0 : (l1 >= l2 ? 1 : 2);
        corr = arg == yy;
        for (int c = 0; c < kOutPad; ++c) {
            const float g = c < 3 ? p[c] - (c == yy ? 1.0f : 0.0f) : 0.0f;
            dL[(long long)b * kOutPad + c] = __float2bfloat16_rn(g);
            dLT[(long long)c * B + b] = __float2bfloat16_rn(g);
        }
    }
    loss = warp_sum(loss);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) corr += __shfl_xor_sync(0xffffffffu, corr, o);
    if ((threadIdx.x & 31) == 0) {
        sl[threadIdx.x >> 5] = loss;
        sc[threadIdx.x >> 5] = corr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tl = 0.0;
        int tc = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            tl += sl[w];
            tc += sc[w];
        }
        loss_part[blockIdx.x] = tl;
        correct_part[blockIdx.x] = tc;
    }
}

// Row sums of a transposed gradient G^T[rows x B] (bias gradients), one
// warp per row, fixed order.
__global__ void rowsum_kernel(const bf16 *GT, int rows, int B, float *out)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= rows) return;
    float s = 0.0f;
    for (int b = lane; b < B; b += 32) s += __bfloat162float(GT[(long long)w * B + b]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[w] = s;
}

// Gradient of one parameter tensor element (o, i) of a [rows x cols]
// weight: sum over splits of the weight-gradient GEMM partials, read
// transposed when the GEMM produced W^T, or a finished sum (biases); times
// 1/B (the loss kernel leaves dL unscaled).
struct GradSrc {
    const float *part;  // [splits][prow x pcol] GEMM partials, or null
    const float *gsum;  // finished sums, or null
    int splits, prow, pcol;
    int transposed;
    int rows, cols;
};

__device__ __forceinline__ float grad_of(const GradSrc &g, int idx, float inv_b)
{
    const int o = idx / g.cols, i = idx % g.cols;
    float s = 0.0f;
    if (g.part) {
        const long long off = g.transposed ? (long long)i * g.pcol + o : (long long)o * g.pcol + i;
        for (int k = 0; k < g.splits; ++k) s += g.part[(long long)k * g.prow * g.pcol + off];
    } else {
        s = g.gsum[idx];
    }
    return s * inv_b;
}

// AdamW (decoupled weight decay) on FP32 master weights; refreshes the BF16
// copy W (row-major [rows x cols]) and W^T ([cols x ldt]) used by the GEMMs.
struct AdamArgs {
    GradSrc g;
    float *w, *m, *v;
    __nv_bfloat16 *wb, *wbT;
    float *fcopy;  // FP32 copy (padded bias of the logits), or null
    int ldt;
    float inv_b, lr, wd, b1, b2, eps, c1, c2;  // c1 = 1/(1-b1^t), c2 = 1/(1-b2^t)
};

__global__ void adamw_kernel(const AdamArgs a)
{
    const int n = a.g.rows * a.g.cols;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        const float g = grad_of(a.g, idx, a.inv_b);
        const float m = a.b1 * a.m[idx] + (1.0f - a.b1) * g;
        const float v = a.b2 * a.v[idx] + (1.0f - a.b2) * g * g;
        a.m[idx] = m;
        a.v[idx] = v;
        float w = a.w[idx];
        w -= a.lr * ((m * a.c1) / (sqrtf(v * a.c2) + a.eps) + a.wd * w);
        a.w[idx] = w;
        const int o = idx / a.g.cols, i = idx % a.g.cols;
        const __nv_bfloat16 wb = __float2bfloat16_rn(w);
        if (a.wb) a.wb[idx] = wb;
        if (a.wbT) a.wbT[(long long)i * a.ldt + o] = wb;
        if (a.fcopy) a.fcopy[idx] = w;
    }
}

__global__ void grad_kernel(const GradSrc g, float inv_b, float *out)
{
    const int n = g.rows * g.cols;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x)
        out[idx] = grad_of(g, idx, inv_b);
}

// argmax of the 3 logits -> indicator tag (class index)
__global__ void argmax_kernel(const float *L, int B, int *cls)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float l0 = L[(long long)b * kOutPad], l1 = L[(long long)b * kOutPad + 1], l2 = L[(long long)b * kOutPad + 2];
    cls[b] = (l0 >= l1 && l0 >= l2) ? 0 : (l1 >= l2 ? 1 : 2);
}

// plain three-class label from the jump: refine (1) when J >= tol, coarsen
// (0) when J < lo_frac * tol, keep (2) in between. cover: merged into the
// label already there, keeping the finer demand (refine if either asks for
// it, coarsen only if both do, keep otherwise)
__global__ void label_kernel(const double *J, int n, double tol, double lo_frac, int *cls, int cover)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double j = J[k];
    int c = j >= tol ? kClassRefine : (j < lo_frac * tol ? kClassCoarsen : kClassKeep);
    if (cover) {
        const int old = cls[k];
        c = (old == kClassRefine || c == kClassRefine) ? kClassRefine
            : (old == kClassCoarsen && c == kClassCoarsen) ? kClassCoarsen : kClassKeep;
    }
    cls[k] = c;
}

// ---------------------------------------------------------------- host side

static int grid1(long long n, int block) { return (int)std::max<long long>(1, std::min<long long>((n + block - 1) / block, 148LL * 32)); }

cudaError_t mlp_launch_features(int n, const double *q, long long stride, const QuadDesc *quads, int nquad, bf16 *X,
                                cudaStream_t st)
{
    if (nquad <= 0) return cudaSuccess;
    switch (n) {
    case 8: features_kernel<8><<<nquad, 128, 0, st>>>(q, stride, quads, nquad, X); break;
    case 16: features_kernel<16><<<nquad, 128, 0, st>>>(q, stride, quads, nquad, X); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t mlp_launch_jump(int n, const double *rho, const QuadDesc *quads, const int *which, int count, double *J,
                            cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    const int blocks = (count * 32 + 255) / 256;
    switch (n) {
    case 2: jump_kernel<2><<<blocks, 256, 0, st>>>(rho, quads, which, count, J); break;
    case 4: jump_kernel<4><<<blocks, 256, 0, st>>>(rho, quads, which, count, J); break;
    case 8: jump_kernel<8><<<blocks, 256, 0, st>>>(rho, quads, which, count, J); break;
    case 16: jump_kernel<16><<<blocks, 256, 0, st>>>(rho, quads, which, count, J); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t mlp_launch_labels(const double *J, int n, double tol, double lo_frac, int *cls, cudaStream_t st,
                              bool cover)
{
    if (n <= 0) return cudaSuccess;
    label_kernel<<<(n + 255) / 256, 256, 0, st>>>(J, n, tol, lo_frac, cls, cover ? 1 : 0);
    return cudaGetLastError();
}

namespace {

template <typename T>
bool dalloc(T **p, size_t n, std::vector<void *> &own)
{
    if (cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess) return false;
    own.push_back((void *)*p);
    return true;
}

// Offsets of the flat FP32 parameter vector: W1 [128x400], b1, W2 [64x128],
// b2, W3 [3x64], b3.
const int kParamOff[7] = {0,
                          kH1 * kFeatIn,
                          kH1 * kFeatIn + kH1,
                          kH1 * kFeatIn + kH1 + kH2 * kH1,
                          kH1 * kFeatIn + kH1 + kH2 * kH1 + kH2,
                          kH1 * kFeatIn + kH1 + kH2 * kH1 + kH2 + kOut * kH2,
                          kMlpParams};

}  // namespace

MlpState::~MlpState() { release(); }

void MlpState::release()
{
    for (void *p : batch_owned) cudaFree(p);
    for (void *p : fixed_owned) cudaFree(p);
    batch_owned.clear();
    fixed_owned.clear();
    cudaFree(Xall);
    cudaFree(yall);
    cudaFree(perm);
    cudaFree(jump);
    cudaFree(which);
    cudaFree(jcls);
    Xall = nullptr;
    yall = nullptr;
    perm = nullptr;
    jump = nullptr;
    which = nullptr;
    jcls = nullptr;
    cap_batch = 0;
    cap_data = n_data = cap_perm = 0;
    cap_judge = 0;
}

bool MlpState::init(uint64_t seed)
{
    auto &o = fixed_owned;
    if (!dalloc(&w, kMlpParams, o) || !dalloc(&m, kMlpParams, o) || !dalloc(&v, kMlpParams, o) ||
        !dalloc(&W1, size_t(kH1) * kFeatIn, o) || !dalloc(&W2, size_t(kH2) * kH1, o) ||
        !dalloc(&W3, size_t(kOutPad) * kH2, o) || !dalloc(&W2T, size_t(kH1) * kH2, o) ||
        !dalloc(&W3T, size_t(kH2) * kOutPad, o) || !dalloc(&b3p, kOutPad, o) || !dalloc(&err, 1, o))
        return false;
    // deterministic init: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and
    // biases, from splitmix64 of the seed and the element index
    std::vector<float> h(kMlpParams);
    auto u01 = [&](uint64_t k) {
        uint64_t z = seed * 0x9E3779B97F4A7C15ULL + k + 0x632BE59BD9B4E019ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    const int fan[6] = {kFeatIn, kFeatIn, kH1, kH1, kH2, kH2};
    for (int t = 0; t < 6; ++t)
        for (int k = kParamOff[t]; k < kParamOff[t + 1]; ++k)
            h[size_t(k)] = (float)((2.0 * u01(uint64_t(k)) - 1.0) / std::sqrt((double)fan[t]));
    return set_params(h.data());
}

bool MlpState::set_params(const float *h)
{
    if (cudaMemcpy(w, h, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice) != cudaSuccess) return false;
    if (cudaMemset(m, 0, sizeof(float) * kMlpParams) != cudaSuccess) return false;
    if (cudaMemset(v, 0, sizeof(float) * kMlpParams) != cudaSuccess) return false;
    step = 0;
    return refresh_bf16();
}

// BF16 GEMM copies of the FP32 master weights (host round trip; set-up only)
bool MlpState::refresh_bf16()
{
    using bf = __nv_bfloat16;
    std::vector<float> h(kMlpParams);
    if (cudaMemcpy(h.data(), w, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    const bf zero = __float2bfloat16(0.0f);
    std::vector<bf> w1(size_t(kH1) * kFeatIn), w2(size_t(kH2) * kH1), w3(size_t(kOutPad) * kH2, zero),
        w2t(size_t(kH1) * kH2), w3t(size_t(kH2) * kOutPad, zero);
    std::vector<float> b3(kOutPad, 0.0f);
    for (int k = 0; k < kH1 * kFeatIn; ++k) w1[size_t(k)] = __float2bfloat16(h[size_t(kParamOff[0] + k)]);
    for (int o = 0; o < kH2; ++o)
        for (int i = 0; i < kH1; ++i) {
            const bf b = __float2bfloat16(h[size_t(kParamOff[2] + o * kH1 + i)]);
            w2[size_t(o * kH1 + i)] = b;
            w2t[size_t(i * kH2 + o)] = b;
        }
    for (int o = 0; o < kOut; ++o) {
        for (int i = 0; i < kH2; ++i) {
            const bf b = __float2bfloat16(h[size_t(kParamOff[4] + o * kH2 + i)]);
            w3[size_t(o * kH2 + i)] = b;
            w3t[size_t(i * kOutPad + o)] = b;
        }
        b3[size_t(o)] = h[size_t(kParamOff[5] + o)];
    }
    return cudaMemcpy(W1, w1.data(), w1.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(W2, w2.data(), w2.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(W3, w3.data(), w3.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(W2T, w2t.data(), w2t.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(W3T, w3t.data(), w3t.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(b3p, b3.data(), b3.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemset(err, 0, sizeof(int)) == cudaSuccess;
}

bool MlpState::ensure_batch(int B)
{
    if (B <= cap_batch) return true;
    // twice the old capacity at least (rows stay a multiple of 128): a mesh
    // that grows a few quads per regrid reallocates rarely
    B = std::max(B, 2 * cap_batch);
    cudaStreamSynchronize(stream);
    for (void *p : batch_owned) cudaFree(p);
    batch_owned.clear();
    cap_batch = 0;
    auto &o = batch_owned;
    const size_t b = size_t(B);
    const size_t splits = (b + kWgradK - 1) / kWgradK;
    const size_t blocks = (b + 255) / 256;
    const bool ok =
        dalloc(&X, b * kFeatIn, o) && dalloc(&XT, b * kFeatIn, o) && dalloc(&y, b, o) && dalloc(&Z1, b * kH1, o) &&
        dalloc(&H1, b * kH1, o) && dalloc(&H1T, b * kH1, o) && dalloc(&Z2, b * kH2, o) && dalloc(&H2, b * kH2, o) &&
        dalloc(&H2T, b * kH2, o) && dalloc(&Lg, b * kOutPad, o) && dalloc(&dL, b * kOutPad, o) &&
        dalloc(&dLT, b * kOutPad, o) && dalloc(&dZ2, b * kH2, o) && dalloc(&dZ2T, b * kH2, o) &&
        dalloc(&dZ1T, b * kH1, o) && dalloc(&P1, splits * kH1 * kFeatIn, o) && dalloc(&P2, splits * kH1 * kH2, o) &&
        dalloc(&P3, splits * kH2 * kOutPad, o) && dalloc(&gb, size_t(kH1 + kH2 + kOutPad), o) &&
        dalloc(&gflat, size_t(kMlpParams), o) && dalloc(&loss_part, blocks, o) && dalloc(&corr_part, blocks, o) &&
        dalloc(&cls, b, o);
    if (ok) cap_batch = B;
    return ok;
}

bool MlpState::ensure_data(long long n)
{
    if (n <= cap_data) return true;
    long long cap = std::max<long long>(n, cap_data * 2);
    __nv_bfloat16 *nx = nullptr;
    int *ny = nullptr;
    if (cudaMalloc(&nx, sizeof(__nv_bfloat16) * size_t(cap) * kFeatIn) != cudaSuccess) return false;
    if (cudaMalloc(&ny, sizeof(int) * size_t(cap)) != cudaSuccess) {
        cudaFree(nx);
        return false;
    }
    if (n_data > 0) {
        cudaMemcpyAsync(nx, Xall, sizeof(__nv_bfloat16) * size_t(n_data) * kFeatIn, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(ny, yall, sizeof(int) * size_t(n_data), cudaMemcpyDeviceToDevice, stream);
    }
    cudaStreamSynchronize(stream);
    cudaFree(Xall);
    cudaFree(yall);
    Xall = nx;
    yall = ny;
    cap_data = cap;
    return true;
}

bool MlpState::ensure_judge(int n)
{
    if (n <= cap_judge) return true;
    n = std::max(2 * n, 1024);  // headroom: the judged quads follow the mesh
    cudaStreamSynchronize(stream);
    cudaFree(jump);
    cudaFree(which);
    cudaFree(jcls);
    jump = nullptr;
    which = jcls = nullptr;
    cap_judge = 0;
    if (cudaMalloc(&jump, sizeof(double) * size_t(n)) != cudaSuccess ||
        cudaMalloc(&which, sizeof(int) * size_t(n)) != cudaSuccess ||
        cudaMalloc(&jcls, sizeof(int) * size_t(n)) != cudaSuccess)
        return false;
    cap_judge = n;
    return true;
}

// Forward pass of B rows of X (device, row-major): logits into Lg; with
// `train` also Z1, Z2, H1^T, H2^T for the backward pass.
cudaError_t MlpState::forward(int B, bool train, cudaStream_t st)
{
    GemmArgs g{};
    g.err = err;
    // fwd1: [B x 400] x W1[128 x 400]^T
    g.A = X; g.lda = kFeatIn; g.B = W1; g.ldb = kFeatIn; g.M = B; g.N = kH1; g.K = kFeatIn; g.k_per_split = kFeatIn;
    g.bias = w + kParamOff[1]; g.zout = train ? Z1 : nullptr; g.hout = H1; g.houtT = train ? H1T : nullptr; g.ldt = B;
    cudaError_t e = launch_gemm<128, kEpiHidden>(g, 1, st);
    if (e != cudaSuccess) return e;
    // fwd2: [B x 128] x W2[64 x 128]^T
    g.A = H1; g.lda = kH1; g.B = W2; g.ldb = kH1; g.N = kH2; g.K = kH1; g.k_per_split = kH1;
    g.bias = w + kParamOff[3]; g.zout = train ? Z2 : nullptr; g.hout = H2; g.houtT = train ? H2T : nullptr;
    if ((e = launch_gemm<64, kEpiHidden>(g, 1, st)) != cudaSuccess) return e;
    // fwd3: [B x 64] x W3[16 x 64]^T (rows 3..15 zero)
    g.A = H2; g.lda = kH2; g.B = W3; g.ldb = kH2; g.N = kOutPad; g.K = kH2; g.k_per_split = kH2;
    g.bias = b3p; g.zout = Lg; g.hout = nullptr; g.houtT = nullptr;
    return launch_gemm<16, kEpiLogits>(g, 1, st);
}

cudaError_t MlpState::loss(int B, cudaStream_t st)
{
    softmax_ce_kernel<<<(B + 255) / 256, 256, 0, st>>>(Lg, y, B, dL, dLT, loss_part, corr_part);
    return cudaGetLastError();
}

// Backward pass after forward(B, true) and loss(B): the weight-gradient
// partials P1..P3 and the bias sums gb.
cudaError_t MlpState::backward(int B, cudaStream_t st)
{
    GemmArgs g{};
    g.err = err;
    // bwd3: dH2 = dL[B x 16] W3p[16 x 64]; operand W3^T[64 x 16]
    g.A = dL; g.lda = kOutPad; g.B = W3T; g.ldb = kOutPad; g.M = B; g.N = kH2; g.K = kOutPad; g.k_per_split = kOutPad;
    g.zin = Z2; g.hout = dZ2; g.houtT = dZ2T; g.ldt = B;
    cudaError_t e = launch_gemm<64, kEpiBackHidden>(g, 1, st);
    if (e != cudaSuccess) return e;
    // bwd2: dH1 = dZ2[B x 64] W2[64 x 128]; operand W2^T[128 x 64]
    g.A = dZ2; g.lda = kH2; g.B = W2T; g.ldb = kH2; g.N = kH1; g.K = kH2; g.k_per_split = kH2;
    g.zin = Z1; g.hout = nullptr; g.houtT = dZ1T;
    if ((e = launch_gemm<128, kEpiBackHidden>(g, 1, st)) != cudaSuccess) return e;
    // weight gradients, K = batch in slices of kWgradK rows
    const int splits = (B + kWgradK - 1) / kWgradK;
    GemmArgs p{};
    p.err = err;
    p.k_per_split = kWgradK;
    p.K = B;
    // dW1[128 x 400] = dZ1^T[128 x B] (X^T[400 x B])^T
    p.A = dZ1T; p.lda = B; p.B = XT; p.ldb = B; p.M = kH1; p.N = kFeatIn; p.zout = P1;
    if ((e = launch_gemm<80, kEpiPartial>(p, splits, st)) != cudaSuccess) return e;
    // dW2^T[128 x 64] = H1^T[128 x B] (dZ2^T[64 x B])^T
    p.A = H1T; p.B = dZ2T; p.M = kH1; p.N = kH2; p.zout = P2;
    if ((e = launch_gemm<64, kEpiPartial>(p, splits, st)) != cudaSuccess) return e;
    // dW3^T[64 x 16] = H2^T[64 x B] (dL^T[16 x B])^T
    p.A = H2T; p.B = dLT; p.M = kH2; p.N = kOutPad; p.zout = P3;
    if ((e = launch_gemm<16, kEpiPartial>(p, splits, st)) != cudaSuccess) return e;
    // bias gradients: row sums of dZ1^T, dZ2^T, dL^T
    rowsum_kernel<<<(kH1 * 32 + 255) / 256, 256, 0, st>>>(dZ1T, kH1, B, gb);
    rowsum_kernel<<<(kH2 * 32 + 255) / 256, 256, 0, st>>>(dZ2T, kH2, B, gb + kH1);
    rowsum_kernel<<<(kOutPad * 32 + 255) / 256, 256, 0, st>>>(dLT, kOutPad, B, gb + kH1 + kH2);
    return cudaGetLastError();
}

namespace {

// where each parameter tensor's gradient lives after backward()
GradSrc grad_src(const MlpState &s, int t, int B)
{
    const int splits = (B + kWgradK - 1) / kWgradK;
    GradSrc g{};
    g.splits = splits;
    switch (t) {
    case 0: g.part = s.P1; g.prow = kH1; g.pcol = kFeatIn; g.rows = kH1; g.cols = kFeatIn; break;
    case 1: g.gsum = s.gb; g.rows = 1; g.cols = kH1; break;
    case 2: g.part = s.P2; g.prow = kH1; g.pcol = kH2; g.transposed = 1; g.rows = kH2; g.cols = kH1; break;
    case 3: g.gsum = s.gb + kH1; g.rows = 1; g.cols = kH2; break;
    case 4: g.part = s.P3; g.prow = kH2; g.pcol = kOutPad; g.transposed = 1; g.rows = kOut; g.cols = kH2; break;
    default: g.gsum = s.gb + kH1 + kH2; g.rows = 1; g.cols = kOut; break;
    }
    return g;
}

}  // namespace

cudaError_t MlpState::update(int B, float lr, float wd, cudaStream_t st)
{
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    AdamArgs a{};
    a.inv_b = 1.0f / (float)B;
    a.lr = lr;
    a.b1 = b1;
    a.b2 = b2;
    a.eps = 1e-8f;
    a.c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)step)));
    a.c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)step)));
    for (int t = 0; t < 6; ++t) {
        a.g = grad_src(*this, t, B);
        a.w = w + kParamOff[t];
        a.m = m + kParamOff[t];
        a.v = v + kParamOff[t];
        a.wd = (t % 2 == 0) ? wd : 0.0f;  // no decay on biases
        a.wb = t == 0 ? W1 : t == 2 ? W2 : t == 4 ? W3 : nullptr;
        a.wbT = t == 2 ? W2T : t == 4 ? W3T : nullptr;
        a.ldt = t == 2 ? kH2 : kOutPad;
        a.fcopy = t == 5 ? b3p : nullptr;
        const long long n = (long long)a.g.rows * a.g.cols;
        adamw_kernel<<<grid1(n, 256), 256, 0, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t MlpState::flat_grad(int B, cudaStream_t st)
{
    for (int t = 0; t < 6; ++t) {
        const GradSrc g = grad_src(*this, t, B);
        grad_kernel<<<grid1((long long)g.rows * g.cols, 256), 256, 0, st>>>(g, 1.0f / (float)B, gflat + kParamOff[t]);
    }
    return cudaGetLastError();
}

cudaError_t MlpState::gather(const int *perm_dev, int b0, int B, cudaStream_t st)
{
    gather_kernel<<<B, 128, 0, st>>>(Xall, yall, perm_dev, b0, B, X, XT, y);
    return cudaGetLastError();
}

cudaError_t MlpState::argmax(int B, int *out, cudaStream_t st)
{
    argmax_kernel<<<(B + 255) / 256, 256, 0, st>>>(Lg, B, out);
    return cudaGetLastError();
}

}  // namespace amrgpu
