// se_hoststage.cu -- copies between the caller's pageable host arrays and
// device memory for the reference-API entry points (se_legacy.cu,
// se_fftw.cu), which take malloc'd host arrays and must leave their results
// there before they return.
//
// A plain cudaMemcpy from pageable memory goes through one driver thread and
// its own bounce buffer: ~10 GB/s host to device on the B200 machines, and
// ~3.6 GB/s device to host into freshly malloc'd arrays (each first touch of
// a page faults on that one thread).  Here a copy is cut into chunks of
// STAGE_CHUNK bytes that alternate between two pinned buffers: host threads
// copy chunk k between the caller's array and one pinned buffer (and take
// the page faults in parallel) while the DMA engine moves chunk k - 1 or
// k + 1 through the other on a stream of its own.  Arrays that are pinned
// already (cudaHostAlloc / cudaHostRegister) go straight through
// cudaMemcpy, and so does everything if the pinned buffers cannot be had.
//
// Both directions return when the data is in place: host_to_device after
// its stream drained (so work launched afterwards on any stream sees the
// data), device_to_host after the last chunk was copied out.  device_to_host
// must be called after the device work that wrote the source has finished
// (the callers synchronise the device first).  One copy runs at a time per
// process (a mutex); the buffers, stream and events belong to the device
// that was current at the first copy of each device.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "se_internal.h"

namespace se {
namespace {

constexpr size_t STAGE_CHUNK = size_t(4) << 20;   // bytes per pinned buffer
constexpr size_t STAGE_MIN = size_t(1) << 20;     // smaller copies: cudaMemcpy
constexpr size_t SLICE_MIN = size_t(256) << 10;   // per host thread and chunk

// Splits one memcpy over the pool's threads and the calling thread.
class CopyPool {
public:
    CopyPool()
    {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        nthreads_ = (int)std::min(7u, std::max(1u, hw / 2) - 1);
        for (int i = 0; i < nthreads_; i++) std::thread([this] { worker(); }).detach();
    }

    void copy(void* dst, const void* src, size_t n)
    {
        const int parts = (int)std::min<size_t>(nthreads_ + 1, std::max<size_t>(1, n / SLICE_MIN));
        if (parts <= 1) {
            memcpy(dst, src, n);
            return;
        }
        std::unique_lock<std::mutex> l(mu_);
        dst_ = static_cast<char*>(dst);
        src_ = static_cast<const char*>(src);
        bytes_ = n;
        slice_ = ((n + parts - 1) / parts + 63) & ~size_t(63);
        nslices_ = (int)((n + slice_ - 1) / slice_);
        next_ = 0;
        done_ = 0;
        job_++;
        cv_work_.notify_all();
        run(l);
        cv_done_.wait(l, [&] { return done_ == nslices_; });
    }

private:
    // Takes slices of the current job until none is left (mu_ held on entry
    // and exit, released around each memcpy).
    void run(std::unique_lock<std::mutex>& l)
    {
        while (next_ < nslices_) {
            const size_t off = (size_t)(next_++) * slice_;
            const size_t len = std::min(slice_, bytes_ - off);
            char* d = dst_ + off;
            const char* s = src_ + off;
            l.unlock();
            memcpy(d, s, len);
            l.lock();
            if (++done_ == nslices_) cv_done_.notify_all();
        }
    }

    void worker()
    {
        unsigned long long seen = 0;
        std::unique_lock<std::mutex> l(mu_);
        for (;;) {
            cv_work_.wait(l, [&] { return job_ != seen; });
            seen = job_;
            run(l);
        }
    }

    int nthreads_ = 0;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    unsigned long long job_ = 0;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t bytes_ = 0, slice_ = 0;
    int nslices_ = 0, next_ = 0, done_ = 0;
};

struct DeviceStage {
    void* pin[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool ok = false;
};

std::mutex g_mu;   // one staged copy at a time

CopyPool& pool()
{
    static CopyPool* p = new CopyPool();   // threads live until the process exits
    return *p;
}

DeviceStage* stage_for_current_device()
{
    static std::map<int, DeviceStage>* m = new std::map<int, DeviceStage>();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    auto it = m->find(dev);
    if (it != m->end()) return it->second.ok ? &it->second : nullptr;
    DeviceStage& s = (*m)[dev];
    s.ok = cudaHostAlloc(&s.pin[0], STAGE_CHUNK, cudaHostAllocDefault) == cudaSuccess &&
           cudaHostAlloc(&s.pin[1], STAGE_CHUNK, cudaHostAllocDefault) == cudaSuccess &&
           cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&s.ev[0], cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&s.ev[1], cudaEventDisableTiming) == cudaSuccess;
    if (!s.ok) cudaGetLastError();   // stay on cudaMemcpy; clear the error
    return s.ok ? &s : nullptr;
}

}  // namespace

bool host_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

int host_to_device(void* d, const void* h, size_t n)
{
    if (n == 0) return SE_OK;
    if (n < STAGE_MIN || host_pinned(h)) {
        SE_CUDA(cudaMemcpy(d, h, n, cudaMemcpyHostToDevice));
        return SE_OK;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceStage* s = stage_for_current_device();
    if (!s) {
        SE_CUDA(cudaMemcpy(d, h, n, cudaMemcpyHostToDevice));
        return SE_OK;
    }
    const char* src = static_cast<const char*>(h);
    char* dst = static_cast<char*>(d);
    const size_t nk = (n + STAGE_CHUNK - 1) / STAGE_CHUNK;
    for (size_t k = 0; k < nk; k++) {
        const int b = (int)(k & 1);
        const size_t off = k * STAGE_CHUNK, len = std::min(STAGE_CHUNK, n - off);
        if (k >= 2) SE_CUDA(cudaEventSynchronize(s->ev[b]));   // chunk k - 2 has left it
        pool().copy(s->pin[b], src + off, len);
        SE_CUDA(cudaMemcpyAsync(dst + off, s->pin[b], len, cudaMemcpyHostToDevice, s->st));
        SE_CUDA(cudaEventRecord(s->ev[b], s->st));
    }
    SE_CUDA(cudaStreamSynchronize(s->st));
    return SE_OK;
}

int device_to_host(void* h, const void* d, size_t n)
{
    if (n == 0) return SE_OK;
    if (n < STAGE_MIN || host_pinned(h)) {
        SE_CUDA(cudaMemcpy(h, d, n, cudaMemcpyDeviceToHost));
        return SE_OK;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceStage* s = stage_for_current_device();
    if (!s) {
        SE_CUDA(cudaMemcpy(h, d, n, cudaMemcpyDeviceToHost));
        return SE_OK;
    }
    const char* src = static_cast<const char*>(d);
    char* dst = static_cast<char*>(h);
    const size_t nk = (n + STAGE_CHUNK - 1) / STAGE_CHUNK;
    auto issue = [&](size_t k) -> int {
        const int b = (int)(k & 1);
        const size_t off = k * STAGE_CHUNK, len = std::min(STAGE_CHUNK, n - off);
        SE_CUDA(cudaMemcpyAsync(s->pin[b], src + off, len, cudaMemcpyDeviceToHost, s->st));
        SE_CUDA(cudaEventRecord(s->ev[b], s->st));
        return SE_OK;
    };
    SE_TRY(issue(0));
    for (size_t k = 0; k < nk; k++) {
        // buffer (k + 1) & 1 held chunk k - 1, copied out already
        if (k + 1 < nk) SE_TRY(issue(k + 1));
        const int b = (int)(k & 1);
        const size_t off = k * STAGE_CHUNK, len = std::min(STAGE_CHUNK, n - off);
        SE_CUDA(cudaEventSynchronize(s->ev[b]));
        pool().copy(dst + off, s->pin[b], len);
    }
    return SE_OK;
}

}  // namespace se
