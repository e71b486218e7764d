// se_internal.h -- declarations shared by the translation units of libse_gpu.so.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstdio>

#include "se_gpu.h"

namespace se {

// Records the first CUDA failure of a call chain and returns the SE code.
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define SE_CUDA(call)                                                         \
    do {                                                                      \
        cudaError_t se_e_ = (call);                                           \
        if (se_e_ != cudaSuccess)                                             \
            return ::se::cuda_fail(se_e_, #call, __FILE__, __LINE__);         \
    } while (0)

#define SE_TRY(call)                                                          \
    do {                                                                      \
        int se_r_ = (call);                                                   \
        if (se_r_ != SE_OK) return se_r_;                                     \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline unsigned ceil_div(long a, long b) { return static_cast<unsigned>((a + b - 1) / b); }

// ---- stable counting sort (se_sort.cu) ----
size_t sort_scratch_bytes(int N, int nkeys);
// Sorts (key, value) pairs by key, stably.  vals_in may be NULL (identity).
// Results: perm (the values in key order) and, when offsets != NULL, the
// bin starts offsets[nkeys + 1].  launches is incremented per kernel.
int stable_sort(const int* keys, const int* vals_in, int N, int nkeys, int* perm,
                int* sorted_keys, int* offsets, void* scratch, size_t scratch_bytes,
                cudaStream_t st, int* launches);

// ---- copies between pageable host arrays and device memory (se_hoststage.cu):
// pipelined through pinned chunks, host side split over threads; both return
// when the data is in place.  device_to_host needs the device work that
// wrote d finished.
int host_to_device(void* d, const void* h, size_t bytes);
int device_to_host(void* h, const void* d, size_t bytes);
// p is page-locked host memory (cudaHostAlloc / cudaHostRegister)
bool host_pinned(const void* p);

// Device flag a plan's kernels set when a position was not finite (reset at
// the start of each solve on the plan's stream).
const int* plan_error_flag(se_plan p);

// exclusive scan of n ints (in place allowed), total written to out[n] if
// write_total; scratch of scan_scratch_bytes(n)
size_t scan_scratch_bytes(long n);
int exclusive_scan(const int* in, int* out, long n, bool write_total, void* scratch,
                   cudaStream_t st, int* launches);

}  // namespace se
