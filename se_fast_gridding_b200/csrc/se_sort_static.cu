// se_sort_static.cu -- the stable counting sort with its scratch in a
// file-scope device array: an entry point that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they need the
// sort: code running while a memory pool is frozen or being captured, host
// callbacks and real-time loops that must not block on the allocator, or a
// host library linked into a process whose allocator it does not own.  This
// variant takes only the caller's inputs and outputs; its working memory is
// g_sort_scratch below, SE_SORT_STATIC_BYTES bytes that every GPU which loads
// the library holds until the process exits.
//
// Set-up: the first call on each device looks up the device address of
// g_sort_scratch with cudaGetSymbolAddress (with that device current) and
// caches it for the life of the process; make that first call outside any
// stream capture.  The cache assumes the device's primary context lives as
// long as the process: after a cudaDeviceReset the cached address would
// belong to a context that no longer exists.  All calls
// share the array, which keeps the previous call's contents: the sort clears
// the parts that must start at zero (the bin counts) itself, and calls whose
// work overlaps on the GPU (different streams, concurrent graphs) race on the
// array and must be serialised by the caller.
#include <mutex>

#include "se_internal.h"

namespace {

__device__ __align__(256) unsigned char g_sort_scratch[SE_SORT_STATIC_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void* g_scratch_dev[MAX_DEVICES] = {nullptr};

int scratch_address(void** out)
{
    int dev = 0;
    SE_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return SE_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        SE_CUDA(cudaGetSymbolAddress(&p, g_sort_scratch));
        g_scratch_dev[dev] = p;
    }
    *out = g_scratch_dev[dev];
    return SE_OK;
}

}  // namespace

extern "C" int se_counting_sort_static(const int* keys, int N, int nkeys, int* perm,
                                       int* offsets, void* stream)
{
    if (N < 0 || nkeys < 1 || (N > 0 && (!keys || !perm)) || !offsets) return SE_ERR_INVALID;
    if (N > SE_SORT_STATIC_MAX_N || nkeys > SE_SORT_STATIC_MAX_KEYS) {
        fprintf(stderr,
                "[se_gpu] se_counting_sort_static: N = %d, nkeys = %d exceed the static "
                "scratch limits (N <= %d, nkeys <= %d)\n",
                N, nkeys, SE_SORT_STATIC_MAX_N, SE_SORT_STATIC_MAX_KEYS);
        return SE_ERR_INVALID;
    }
    const size_t need = se::sort_scratch_bytes(N, nkeys);
    if (need > SE_SORT_STATIC_BYTES) return SE_ERR_INVALID;
    void* scratch = nullptr;
    SE_TRY(scratch_address(&scratch));
    return se::stable_sort(keys, nullptr, N, nkeys, perm, nullptr, offsets, scratch, need,
                           se::as_stream(stream), nullptr);
}
