// mlp_internal.h -- the learned indicator's device state and launchers
// (mlp.cu), shared with the C ABI in mlp_api.cu. Not part of the public ABI.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace amrgpu {

struct QuadDesc;

constexpr int kFeatIn = 400;   // 4 fields x 10 x 10 (8 x 8 patch + ring)
constexpr int kH1 = 128;
constexpr int kH2 = 64;
constexpr int kOut = 3;        // classes: coarsen, refine, keep
constexpr int kOutPad = 16;    // smallest UMMA N for M = 128
constexpr int kMlpParams = kH1 * kFeatIn + kH1 + kH2 * kH1 + kH2 + kOut * kH2 + kOut;  // 59,779
constexpr int kWgradK = 256;   // batch rows per split of a weight-gradient GEMM
constexpr double kFeatScale = 10.0;

// class index = indicator tag: 0 coarsen candidate, 1 refine, 2 keep
enum : int { kClassCoarsen = 0, kClassRefine = 1, kClassKeep = 2 };

cudaError_t mlp_launch_features(int n, const double *q, long long stride, const QuadDesc *quads, int nquad,
                                __nv_bfloat16 *X, cudaStream_t st);
cudaError_t mlp_launch_jump(int n, const double *rho, const QuadDesc *quads, const int *which, int count, double *J,
                            cudaStream_t st);
cudaError_t mlp_launch_labels(const double *J, int n, double tol, double lo_frac, int *cls, cudaStream_t st,
                              bool cover = false);

struct MlpState {
    // FP32 master parameters and AdamW moments (flat: W1, b1, W2, b2, W3, b3)
    float *w = nullptr, *m = nullptr, *v = nullptr;
    // BF16 GEMM operands: W1[128x400], W2[64x128], W3[16x64] (rows 3.. zero),
    // W2^T[128x64], W3^T[64x16]; padded FP32 b3[16]
    __nv_bfloat16 *W1 = nullptr, *W2 = nullptr, *W3 = nullptr, *W2T = nullptr, *W3T = nullptr;
    float *b3p = nullptr;
    int *err = nullptr;
    long long step = 0;
    std::vector<void *> fixed_owned;

    // per-batch work buffers (capacity cap_batch rows)
    int cap_batch = 0;
    __nv_bfloat16 *X = nullptr, *XT = nullptr, *H1 = nullptr, *H1T = nullptr, *H2 = nullptr, *H2T = nullptr;
    __nv_bfloat16 *dL = nullptr, *dLT = nullptr, *dZ2 = nullptr, *dZ2T = nullptr, *dZ1T = nullptr;
    float *Z1 = nullptr, *Z2 = nullptr, *Lg = nullptr, *P1 = nullptr, *P2 = nullptr, *P3 = nullptr, *gb = nullptr;
    float *gflat = nullptr;
    double *loss_part = nullptr;
    int *corr_part = nullptr, *y = nullptr, *cls = nullptr;
    std::vector<void *> batch_owned;

    // device dataset of (features, plain label) pairs
    __nv_bfloat16 *Xall = nullptr;
    int *yall = nullptr;
    long long n_data = 0, cap_data = 0;
    int *perm = nullptr;
    long long cap_perm = 0;

    // judge / inference scratch
    double *jump = nullptr;
    int *which = nullptr, *jcls = nullptr;
    int cap_judge = 0;

    cudaStream_t stream = nullptr;

    ~MlpState();
    void release();
    bool init(uint64_t seed);
    bool set_params(const float *h);
    bool refresh_bf16();
    bool ensure_batch(int B);
    bool ensure_data(long long n);
    bool ensure_judge(int n);
    cudaError_t gather(const int *perm_dev, int b0, int B, cudaStream_t st);
    cudaError_t forward(int B, bool train, cudaStream_t st);
    cudaError_t loss(int B, cudaStream_t st);
    cudaError_t backward(int B, cudaStream_t st);
    cudaError_t update(int B, float lr, float wd, cudaStream_t st);
    cudaError_t flat_grad(int B, cudaStream_t st);
    cudaError_t argmax(int B, int *out, cudaStream_t st);
};

}  // namespace amrgpu
