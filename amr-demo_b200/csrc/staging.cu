// staging.cu -- host <-> device copies of a session's state when the host
// array is ordinary pageable memory (the reference's driver allocates its
// solution array with P4EST_ALLOC, amr_external.c:268).
//
// A pageable cudaMemcpyAsync goes through the driver's own small bounce
// buffer one piece at a time with the copying thread blocked. Here the
// array moves through a ring of two pinned chunks instead: host threads copy
// chunk k between the caller's array and pinned slot k % 2 while the DMA
// engine moves chunk k - 1, so the transfer runs at about the slower of the
// pinned PCIe rate and the host threads' memcpy rate. Pinned caller arrays
// (cudaHostAlloc / cudaHostRegister) skip the ring.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "amrgpu_internal.h"

namespace amrgpu {

namespace {

// A fixed pool of host threads for the chunk copies (created on first use,
// joined at exit): run(parts, fn) calls fn(0..parts-1) across the pool and
// the calling thread and returns when all are done.
class CopyPool {
public:
    static CopyPool &get()
    {
        static CopyPool pool;
        return pool;
    }
    void run(int parts, const std::function<void(int)> &fn)
    {
        std::unique_lock<std::mutex> lk(run_mu_);  // one job at a time
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &fn;
            parts_ = parts;
            next_ = 0;
            done_ = 0;
            ++generation_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> g(mu_);
        done_cv_.wait(g, [&] { return done_ == parts_; });
        job_ = nullptr;
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
            ++generation_;
        }
        cv_.notify_all();
        for (auto &t : workers_) t.join();
    }

private:
    CopyPool()
    {
        // a quarter of the host's hardware threads (4 on the 16-core hosts
        // measured: the pageable round trip ran at 1.7 / 2.6 / 3.1 / 3.0 /
        // 2.7 / 1.4 G cell-updates/s with 1 / 2 / 4 / 6 / 8 / 16 threads --
        // more threads than that contend for the host's memory bandwidth),
        // the caller included; AMRGPU_COPY_THREADS overrides
        const int hw = std::max(1, int(std::thread::hardware_concurrency()));
        int n = std::min(8, std::max(1, hw / 4)) - 1;
        if (const char *e = std::getenv("AMRGPU_COPY_THREADS")) n = std::max(0, std::atoi(e) - 1);
        n = std::min<int>(n, hw - 1);
        for (int k = 0; k < n; ++k) workers_.emplace_back([this] { loop(); });
    }
    void loop()
    {
        unsigned long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || generation_ != seen; });
                if (stop_) return;
                seen = generation_;
            }
            work();
        }
    }
    // Claims pieces of the current job until none is left. The job and the
    // piece index are taken together under the lock, so a piece always
    // belongs to the job that run() keeps alive until every piece is done.
    void work()
    {
        for (;;) {
            const std::function<void(int)> *job;
            int k;
            {
                std::lock_guard<std::mutex> g(mu_);
                if (!job_ || next_ >= parts_) return;
                job = job_;
                k = next_++;
            }
            (*job)(k);
            std::lock_guard<std::mutex> g(mu_);
            if (++done_ == parts_) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *job_ = nullptr;
    int parts_ = 0, done_ = 0, next_ = 0;
    unsigned long generation_ = 0;
    bool stop_ = false;
};

void parallel_copy(void *dst, const void *src, size_t bytes)
{
    constexpr size_t kPiece = size_t(1) << 20;
    const int parts = int((bytes + kPiece - 1) / kPiece);
    if (parts <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    CopyPool::get().run(parts, [&](int k) {
        const size_t off = size_t(k) * kPiece;
        std::memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off,
                    std::min(kPiece, bytes - off));
    });
}

bool ok(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return true;
    set_error(AMRGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

}  // namespace

bool host_is_pinned(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

bool PinnedRing::ensure()
{
    if (buf[0]) return true;
    for (int k = 0; k < 2; ++k) {
        if (!ok(cudaHostAlloc(&buf[k], kChunk, cudaHostAllocDefault), "cudaHostAlloc ring")) return false;
        cudaEvent_t e = nullptr;
        if (!ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "ring event")) return false;
        ev[k] = e;
    }
    return true;
}

void PinnedRing::release()
{
    for (int k = 0; k < 2; ++k) {
        if (ev[k]) cudaEventDestroy(static_cast<cudaEvent_t>(ev[k]));
        if (buf[k]) cudaFreeHost(buf[k]);
        buf[k] = nullptr;
        ev[k] = nullptr;
    }
}

bool ring_h2d(PinnedRing &r, void *dst, const void *src, size_t bytes, void *stream)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (host_is_pinned(src)) return ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "H2D");
    if (!r.ensure()) return false;
    size_t off = 0;
    for (int k = 0; off < bytes; ++k) {
        const int slot = k & 1;
        const size_t len = std::min(PinnedRing::kChunk, bytes - off);
        // the DMA that last read this slot (chunk k - 2) has finished
        if (!ok(cudaEventSynchronize(static_cast<cudaEvent_t>(r.ev[slot])), "ring wait")) return false;
        parallel_copy(r.buf[slot], static_cast<const char *>(src) + off, len);
        if (!ok(cudaMemcpyAsync(static_cast<char *>(dst) + off, r.buf[slot], len, cudaMemcpyHostToDevice, st),
                "H2D chunk"))
            return false;
        if (!ok(cudaEventRecord(static_cast<cudaEvent_t>(r.ev[slot]), st), "ring record")) return false;
        off += len;
    }
    return true;
}

bool ring_d2h(PinnedRing &r, void *dst, const void *src, size_t bytes, void *stream)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (host_is_pinned(dst)) {
        return ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "D2H") &&
               ok(cudaStreamSynchronize(st), "sync");
    }
    if (!r.ensure()) return false;
    // DMA of chunk k into slot k % 2, then the host copy of chunk k - 1 out
    // of the other slot while it runs
    size_t off = 0, prev_off = 0, prev_len = 0;
    int k = 0;
    for (; off < bytes; ++k) {
        const int slot = k & 1;
        const size_t len = std::min(PinnedRing::kChunk, bytes - off);
        if (!ok(cudaMemcpyAsync(r.buf[slot], static_cast<const char *>(src) + off, len, cudaMemcpyDeviceToHost, st),
                "D2H chunk"))
            return false;
        if (!ok(cudaEventRecord(static_cast<cudaEvent_t>(r.ev[slot]), st), "ring record")) return false;
        if (k > 0) {
            const int ps = slot ^ 1;
            if (!ok(cudaEventSynchronize(static_cast<cudaEvent_t>(r.ev[ps])), "ring wait")) return false;
            parallel_copy(static_cast<char *>(dst) + prev_off, r.buf[ps], prev_len);
        }
        prev_off = off;
        prev_len = len;
        off += len;
    }
    if (k > 0) {
        const int ps = (k - 1) & 1;
        if (!ok(cudaEventSynchronize(static_cast<cudaEvent_t>(r.ev[ps])), "ring wait")) return false;
        parallel_copy(static_cast<char *>(dst) + prev_off, r.buf[ps], prev_len);
    }
    return ok(cudaStreamSynchronize(st), "sync");
}

}  // namespace amrgpu
