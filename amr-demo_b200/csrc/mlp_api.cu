// mlp_api.cu -- C ABI of the learned refinement indicator (declared in
// include/amrgpu.h): model life cycle, the device dataset of (features,
// plain label) pairs, training epochs, the gradient of one batch for the
// CPU gradient check, and the per-regrid learned tags with the plain
// indicator judging a sampled fraction of the quads.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "amrgpu_internal.h"
#include "device_common.cuh"
#include "mlp_internal.h"

using namespace amrgpu;

struct amrgpu_mlp {
    MlpState st;
};

namespace {

bool ok_cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return true;
    set_error(AMRGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

// device error flags raised by a bounded wait inside a GEMM
bool check_flags(MlpState &s)
{
    int f = 0;
    if (!ok_cuda(cudaMemcpy(&f, s.err, sizeof(int), cudaMemcpyDeviceToHost), "mlp flags")) return false;
    if (f) {
        set_error(AMRGPU_ERR_CUDA, "mlp: a tensor-core wait gave up (timeout flag)");
        cudaMemset(s.err, 0, sizeof(int));
        return false;
    }
    return true;
}

// hash of (seed, quad) in [0, 1): the judge's sample
double judge_u01(unsigned long long seed, int q)
{
    uint64_t z = seed * 0x9E3779B97F4A7C15ULL + (uint64_t)q * 0xD1B54A32D192ED03ULL + 0x8CB92BA72F3D8DD7ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" {

int amrgpu_mlp_create(amrgpu_mlp_t **out, unsigned long long seed)
{
    if (!out) return AMRGPU_ERR_ARG;
    *out = nullptr;
    auto *m = new amrgpu_mlp;
    if (!ok_cuda(cudaStreamCreateWithFlags(&m->st.stream, cudaStreamNonBlocking), "mlp stream") || !m->st.init(seed)) {
        set_error(AMRGPU_ERR_CUDA, "mlp: device allocation or upload failed");
        if (m->st.stream) cudaStreamDestroy(m->st.stream);
        delete m;
        return AMRGPU_ERR_CUDA;
    }
    *out = m;
    return AMRGPU_OK;
}

void amrgpu_mlp_destroy(amrgpu_mlp_t *m)
{
    if (!m) return;
    cudaStreamSynchronize(m->st.stream);
    m->st.release();
    cudaStreamDestroy(m->st.stream);
    delete m;
}

int amrgpu_mlp_get_params(amrgpu_mlp_t *m, float *params)
{
    if (!m || !params) return AMRGPU_ERR_ARG;
    cudaStreamSynchronize(m->st.stream);
    return ok_cuda(cudaMemcpy(params, m->st.w, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost), "get params")
               ? AMRGPU_OK
               : AMRGPU_ERR_CUDA;
}

int amrgpu_mlp_set_params(amrgpu_mlp_t *m, const float *params)
{
    if (!m || !params) return AMRGPU_ERR_ARG;
    cudaStreamSynchronize(m->st.stream);
    return m->st.set_params(params) ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

int amrgpu_session_features(amrgpu_session_t *s, uint16_t *features)
{
    SessionView v{};
    if (!session_view(s, &v) || !features) return AMRGPU_ERR_ARG;
    if (v.n != 8 && v.n != 16) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "features: patches of 8x8 or 16x16 cells only");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (v.nquad == 0) return AMRGPU_OK;
    cudaStream_t st = (cudaStream_t)v.stream;
    const size_t bytes = sizeof(__nv_bfloat16) * size_t(v.nquad) * kFeatIn;
    auto *d = static_cast<__nv_bfloat16 *>(session_scratch(s, bytes));
    if (!d) {
        set_error(AMRGPU_ERR_CUDA, "features: scratch allocation failed");
        return AMRGPU_ERR_CUDA;
    }
    bool ok = ok_cuda(mlp_launch_features(v.n, v.q, v.stride, v.quads, v.nquad, d, st), "features kernel") &&
              ok_cuda(cudaMemcpyAsync(features, d, bytes, cudaMemcpyDeviceToHost, st), "D2H features") &&
              ok_cuda(cudaStreamSynchronize(st), "sync");
    session_count_launches(s, 1);
    return ok ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

int amrgpu_session_jumps(amrgpu_session_t *s, double *jumps)
{
    SessionView v{};
    if (!session_view(s, &v) || !jumps) return AMRGPU_ERR_ARG;
    if (v.nquad == 0) return AMRGPU_OK;
    cudaStream_t st = (cudaStream_t)v.stream;
    auto *d = static_cast<double *>(session_scratch(s, sizeof(double) * size_t(v.nquad)));
    if (!d) {
        set_error(AMRGPU_ERR_CUDA, "jumps: scratch allocation failed");
        return AMRGPU_ERR_CUDA;
    }
    bool ok = ok_cuda(mlp_launch_jump(v.n, v.q, v.quads, nullptr, v.nquad, d, st), "jump kernel") &&
              ok_cuda(cudaMemcpyAsync(jumps, d, sizeof(double) * size_t(v.nquad), cudaMemcpyDeviceToHost, st),
                      "D2H jumps") &&
              ok_cuda(cudaStreamSynchronize(st), "sync");
    session_count_launches(s, 1);
    return ok ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

long long amrgpu_mlp_dataset_append(amrgpu_mlp_t *m, amrgpu_session_t *s, double tol, double lo_frac)
{
    SessionView v{};
    if (!m || !session_view(s, &v) || !(tol > 0.0)) return AMRGPU_ERR_ARG;
    if (v.n != 8 && v.n != 16) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "features: patches of 8x8 or 16x16 cells only");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    MlpState &ms = m->st;
    cudaStream_t st = (cudaStream_t)v.stream;
    if (!ok_cuda(cudaStreamSynchronize(ms.stream), "sync")) return AMRGPU_ERR_CUDA;
    if (!ms.ensure_data(ms.n_data + v.nquad) || !ms.ensure_judge(v.nquad)) {
        set_error(AMRGPU_ERR_CUDA, "dataset: device allocation failed");
        return AMRGPU_ERR_CUDA;
    }
    bool ok = ok_cuda(mlp_launch_features(v.n, v.q, v.stride, v.quads, v.nquad, ms.Xall + ms.n_data * kFeatIn, st),
                      "features kernel") &&
              ok_cuda(mlp_launch_jump(v.n, v.q, v.quads, nullptr, v.nquad, ms.jump, st), "jump kernel") &&
              ok_cuda(mlp_launch_labels(ms.jump, v.nquad, tol, lo_frac, ms.yall + ms.n_data, st), "label kernel") &&
              ok_cuda(cudaStreamSynchronize(st), "sync");
    session_count_launches(s, 3);
    if (!ok) return AMRGPU_ERR_CUDA;
    ms.n_data += v.nquad;
    return ms.n_data;
}

namespace {

// the plain classes of the session's current state into the labels of
// rows [first, first + nquad): replacing them, or merged (cover)
int relabel_rows(amrgpu_mlp_t *m, amrgpu_session_t *s, long long first, double tol, double lo_frac, bool cover)
{
    SessionView v{};
    if (!m || !session_view(s, &v) || !(tol > 0.0) || first < 0 || first + v.nquad > m->st.n_data)
        return AMRGPU_ERR_ARG;
    MlpState &ms = m->st;
    cudaStream_t st = (cudaStream_t)v.stream;
    if (!ms.ensure_judge(v.nquad)) return AMRGPU_ERR_CUDA;
    bool ok = ok_cuda(cudaStreamSynchronize(ms.stream), "sync") &&
              ok_cuda(mlp_launch_jump(v.n, v.q, v.quads, nullptr, v.nquad, ms.jump, st), "jump kernel") &&
              ok_cuda(mlp_launch_labels(ms.jump, v.nquad, tol, lo_frac, ms.yall + first, st, cover), "label kernel") &&
              ok_cuda(cudaStreamSynchronize(st), "sync");
    session_count_launches(s, 2);
    return ok ? AMRGPU_OK : AMRGPU_ERR_CUDA;
}

}  // namespace

int amrgpu_mlp_dataset_relabel(amrgpu_mlp_t *m, amrgpu_session_t *s, long long first, double tol, double lo_frac)
{
    return relabel_rows(m, s, first, tol, lo_frac, false);
}

int amrgpu_mlp_dataset_cover(amrgpu_mlp_t *m, amrgpu_session_t *s, long long first, double tol, double lo_frac)
{
    return relabel_rows(m, s, first, tol, lo_frac, true);
}

long long amrgpu_mlp_dataset_size(const amrgpu_mlp_t *m) { return m ? m->st.n_data : 0; }

int amrgpu_mlp_dataset_clear(amrgpu_mlp_t *m)
{
    if (!m) return AMRGPU_ERR_ARG;
    m->st.n_data = 0;
    return AMRGPU_OK;
}

int amrgpu_mlp_dataset_labels(amrgpu_mlp_t *m, int *labels, long long n)
{
    if (!m || !labels || n < 0 || n > m->st.n_data) return AMRGPU_ERR_ARG;
    if (n == 0) return AMRGPU_OK;
    return ok_cuda(cudaMemcpy(labels, m->st.yall, sizeof(int) * size_t(n), cudaMemcpyDeviceToHost), "D2H labels")
               ? AMRGPU_OK
               : AMRGPU_ERR_CUDA;
}

int amrgpu_mlp_train_epoch(amrgpu_mlp_t *m, const int *perm, long long n, int batch, float lr, float weight_decay,
                           double *mean_loss, double *accuracy)
{
    if (!m || !perm || n < 0 || batch < 128 || batch % 128 != 0 || n > m->st.n_data) return AMRGPU_ERR_ARG;
    MlpState &ms = m->st;
    for (long long k = 0; k < n; ++k)
        if (perm[k] < 0 || perm[k] >= ms.n_data) {
            set_error(AMRGPU_ERR_ARG, "train: permutation entry out of range");
            return AMRGPU_ERR_ARG;
        }
    const long long nb = n / batch;
    if (!ms.ensure_batch(batch)) {
        set_error(AMRGPU_ERR_CUDA, "train: device allocation failed");
        return AMRGPU_ERR_CUDA;
    }
    if (n > ms.cap_perm) {
        cudaFree(ms.perm);
        ms.perm = nullptr;
        ms.cap_perm = 0;
        if (!ok_cuda(cudaMalloc(&ms.perm, sizeof(int) * size_t(n)), "perm alloc")) return AMRGPU_ERR_CUDA;
        ms.cap_perm = n;
    }
    cudaStream_t st = ms.stream;
    if (!ok_cuda(cudaMemcpyAsync(ms.perm, perm, sizeof(int) * size_t(n), cudaMemcpyHostToDevice, st), "H2D perm"))
        return AMRGPU_ERR_CUDA;
    const int blocks = (batch + 255) / 256;
    std::vector<double> lp(size_t(blocks) * size_t(std::max<long long>(nb, 1)));
    std::vector<int> cp(lp.size());
    double *d_lp = nullptr;
    int *d_cp = nullptr;
    if (!ok_cuda(cudaMalloc(&d_lp, sizeof(double) * lp.size()), "alloc") ||
        !ok_cuda(cudaMalloc(&d_cp, sizeof(int) * cp.size()), "alloc")) {
        cudaFree(d_lp);
        return AMRGPU_ERR_CUDA;
    }
    bool ok = true;
    for (long long b = 0; b < nb && ok; ++b) {
        ok = ok_cuda(ms.gather(ms.perm, int(b * batch), batch, st), "gather") &&
             ok_cuda(ms.forward(batch, true, st), "forward") && ok_cuda(ms.loss(batch, st), "loss") &&
             ok_cuda(cudaMemcpyAsync(d_lp + b * blocks, ms.loss_part, sizeof(double) * blocks, cudaMemcpyDeviceToDevice,
                                     st),
                     "loss partials") &&
             ok_cuda(cudaMemcpyAsync(d_cp + b * blocks, ms.corr_part, sizeof(int) * blocks, cudaMemcpyDeviceToDevice,
                                     st),
                     "accuracy partials") &&
             ok_cuda(ms.backward(batch, st), "backward") && ok_cuda(ms.update(batch, lr, weight_decay, st), "adamw");
    }
    if (ok && nb > 0)
        ok = ok_cuda(cudaMemcpyAsync(lp.data(), d_lp, sizeof(double) * size_t(nb * blocks), cudaMemcpyDeviceToHost, st),
                     "D2H") &&
             ok_cuda(cudaMemcpyAsync(cp.data(), d_cp, sizeof(int) * size_t(nb * blocks), cudaMemcpyDeviceToHost, st),
                     "D2H");
    if (ok) ok = ok_cuda(cudaStreamSynchronize(st), "sync") && check_flags(ms);
    cudaFree(d_lp);
    cudaFree(d_cp);
    if (!ok) return AMRGPU_ERR_CUDA;
    double tl = 0.0;
    long long tc = 0;
    for (long long k = 0; k < nb * blocks; ++k) {
        tl += lp[size_t(k)];
        tc += cp[size_t(k)];
    }
    const double rows = (double)std::max<long long>(nb * batch, 1);
    if (mean_loss) *mean_loss = tl / rows;
    if (accuracy) *accuracy = (double)tc / rows;
    return AMRGPU_OK;
}

int amrgpu_mlp_grad(amrgpu_mlp_t *m, const uint16_t *features, const int *labels, int batch, float *logits,
                    float *grad, double *mean_loss)
{
    if (!m || !features || !labels || batch <= 0) return AMRGPU_ERR_ARG;
    if (batch % 8 != 0) {
        set_error(AMRGPU_ERR_ARG, "mlp_grad: batch must be a multiple of 8 (the weight-gradient K)");
        return AMRGPU_ERR_ARG;
    }
    for (int k = 0; k < batch; ++k)
        if (labels[k] < 0 || labels[k] > 2) return AMRGPU_ERR_ARG;
    MlpState &ms = m->st;
    if (!ms.ensure_batch(batch)) return AMRGPU_ERR_CUDA;
    cudaStream_t st = ms.stream;
    const size_t fb = sizeof(uint16_t) * size_t(batch) * kFeatIn;
    std::vector<uint16_t> xt(size_t(batch) * kFeatIn);
    for (int b = 0; b < batch; ++b)
        for (int k = 0; k < kFeatIn; ++k) xt[size_t(k) * batch + b] = features[size_t(b) * kFeatIn + k];
    const int blocks = (batch + 255) / 256;
    std::vector<double> lp((size_t)blocks);
    std::vector<float> lg(size_t(batch) * kOutPad);
    bool ok = ok_cuda(cudaMemcpyAsync(ms.X, features, fb, cudaMemcpyHostToDevice, st), "H2D") &&
              ok_cuda(cudaMemcpyAsync(ms.XT, xt.data(), fb, cudaMemcpyHostToDevice, st), "H2D") &&
              ok_cuda(cudaMemcpyAsync(ms.y, labels, sizeof(int) * size_t(batch), cudaMemcpyHostToDevice, st), "H2D") &&
              ok_cuda(ms.forward(batch, true, st), "forward") && ok_cuda(ms.loss(batch, st), "loss") &&
              ok_cuda(ms.backward(batch, st), "backward") && ok_cuda(ms.flat_grad(batch, st), "grad") &&
              ok_cuda(cudaMemcpyAsync(lg.data(), ms.Lg, sizeof(float) * lg.size(), cudaMemcpyDeviceToHost, st), "D2H") &&
              ok_cuda(cudaMemcpyAsync(lp.data(), ms.loss_part, sizeof(double) * lp.size(), cudaMemcpyDeviceToHost, st),
                      "D2H");
    if (ok && grad)
        ok = ok_cuda(cudaMemcpyAsync(grad, ms.gflat, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, st), "D2H");
    if (ok) ok = ok_cuda(cudaStreamSynchronize(st), "sync") && check_flags(ms);
    if (!ok) return AMRGPU_ERR_CUDA;
    if (logits)
        for (int b = 0; b < batch; ++b)
            for (int c = 0; c < kOut; ++c) logits[size_t(b) * kOut + c] = lg[size_t(b) * kOutPad + c];
    if (mean_loss) {
        double t = 0.0;
        for (double x : lp) t += x;
        *mean_loss = t / batch;
    }
    return AMRGPU_OK;
}

int amrgpu_mlp_predict(amrgpu_mlp_t *m, const uint16_t *features, int batch, float *logits)
{
    if (!m || !features || !logits || batch <= 0) return AMRGPU_ERR_ARG;
    MlpState &ms = m->st;
    if (!ms.ensure_batch(batch)) return AMRGPU_ERR_CUDA;
    cudaStream_t st = ms.stream;
    std::vector<float> lg(size_t(batch) * kOutPad);
    bool ok = ok_cuda(cudaMemcpyAsync(ms.X, features, sizeof(uint16_t) * size_t(batch) * kFeatIn,
                                      cudaMemcpyHostToDevice, st),
                      "H2D") &&
              ok_cuda(ms.forward(batch, false, st), "forward") &&
              ok_cuda(cudaMemcpyAsync(lg.data(), ms.Lg, sizeof(float) * lg.size(), cudaMemcpyDeviceToHost, st), "D2H") &&
              ok_cuda(cudaStreamSynchronize(st), "sync") && check_flags(ms);
    if (!ok) return AMRGPU_ERR_CUDA;
    for (int b = 0; b < batch; ++b)
        for (int c = 0; c < kOut; ++c) logits[size_t(b) * kOut + c] = lg[size_t(b) * kOutPad + c];
    return AMRGPU_OK;
}

int amrgpu_session_learned_tags(amrgpu_session_t *s, amrgpu_mlp_t *m, double judge_fraction, unsigned long long seed,
                                double tol, double lo_frac, int *tags, amrgpu_judge_t *judge)
{
    SessionView v{};
    if (!m || !session_view(s, &v) || !tags || !(tol > 0.0)) return AMRGPU_ERR_ARG;
    if (v.n != 8 && v.n != 16) {
        set_error(AMRGPU_ERR_UNSUPPORTED, "learned tags: patches of 8x8 or 16x16 cells only");
        return AMRGPU_ERR_UNSUPPORTED;
    }
    if (judge) *judge = amrgpu_judge_t{0, 0, 0.0, 0};
    if (v.nquad == 0) return AMRGPU_OK;
    MlpState &ms = m->st;
    cudaStream_t st = (cudaStream_t)v.stream;
    if (!ok_cuda(cudaStreamSynchronize(ms.stream), "sync")) return AMRGPU_ERR_CUDA;
    const int B = ((v.nquad + 127) / 128) * 128;
    if (!ms.ensure_batch(B) || !ms.ensure_judge(v.nquad)) {
        set_error(AMRGPU_ERR_CUDA, "learned tags: device allocation failed");
        return AMRGPU_ERR_CUDA;
    }
    // the judge's sample
    std::vector<int> which;
    if (judge_fraction > 0.0)
        for (int q = 0; q < v.nquad; ++q)
            if (judge_u01(seed, q) < judge_fraction) which.push_back(q);
    const int nj = int(which.size());
    std::vector<int> jl((size_t)nj);
    bool ok = ok_cuda(mlp_launch_features(v.n, v.q, v.stride, v.quads, v.nquad, ms.X, st), "features kernel") &&
              ok_cuda(ms.forward(v.nquad, false, st), "forward") && ok_cuda(ms.argmax(v.nquad, ms.cls, st), "argmax") &&
              ok_cuda(cudaMemcpyAsync(tags, ms.cls, sizeof(int) * size_t(v.nquad), cudaMemcpyDeviceToHost, st), "D2H");
    int launches = 5;
    if (ok && nj > 0) {
        ok = ok_cuda(cudaMemcpyAsync(ms.which, which.data(), sizeof(int) * size_t(nj), cudaMemcpyHostToDevice, st),
                     "H2D judge") &&
             ok_cuda(mlp_launch_jump(v.n, v.q, v.quads, ms.which, nj, ms.jump, st), "jump kernel") &&
             ok_cuda(mlp_launch_labels(ms.jump, nj, tol, lo_frac, ms.jcls, st), "label kernel") &&
             ok_cuda(cudaMemcpyAsync(jl.data(), ms.jcls, sizeof(int) * size_t(nj), cudaMemcpyDeviceToHost, st), "D2H");
        launches += 2;
    }
    if (ok) ok = ok_cuda(cudaStreamSynchronize(st), "sync") && check_flags(ms);
    session_count_launches(s, launches);
    if (!ok) return AMRGPU_ERR_CUDA;
    if (judge) {
        int dis = 0, coarser = 0;
        for (int k = 0; k < nj; ++k) {
            const int p = jl[size_t(k)], t = tags[which[size_t(k)]];
            dis += p != t;
            coarser += (p == kClassRefine && t != kClassRefine) || (t == kClassCoarsen && p != kClassCoarsen);
        }
        judge->judged = nj;
        judge->disagree = dis;
        judge->rate = nj ? (double)dis / nj : 0.0;
        judge->coarser = coarser;
    }
    return AMRGPU_OK;
}

}  // extern "C"
