// se_sort.cu -- integer scan and stable counting sort on the GPU.
//
// The spread and interpolation kernels walk particles bin by bin, so every
// solve first sorts particle indices by grid-bin key.  The sort is a stable
// LSD radix sort with 8-bit digits: per pass a tile histogram, one exclusive
// scan over the digit-major histogram, and a scatter in which each item's rank
// among equal digits is built from (earlier tiles, earlier rounds, earlier
// warps, earlier lanes) only.  The permutation therefore equals the one of a
// CPU stable counting sort, bit for bit, independent of scheduling.  This is
// the GPU counterpart of SE_FGG_reorder_system's qsort (SE_fgg.c:5894-5932),
// with ties kept in input order.
#include "se_internal.h"

namespace se {

namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr long SCAN_BLOCK_MAX = 16L * SCAN_TILE;   // scanned by one block

constexpr int RADIX_BITS = 8;
constexpr int RADIX = 1 << RADIX_BITS;
constexpr int SORT_THREADS = 256;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_ROUNDS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ROUNDS;

size_t align_up(size_t b) { return (b + 255) & ~size_t(255); }

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of one SCAN_TILE tile; tile total to tile_sums / total_out.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(const int* __restrict__ in,
                                                            int* out, long n,
                                                            int* tile_sums, int* total_out)
{
    __shared__ int wsum[SCAN_THREADS / 32];
    const long idx = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int t = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = (idx + i < n) ? in[idx + i] : 0;
        t += v[i];
    }
    const int incl = warp_incl_scan(t);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int s = wsum[lane];
        const int si = warp_incl_scan(s);
        wsum[lane] = si - s;
    }
    __syncthreads();
    const int excl = incl - t + wsum[warp];
    int run = excl;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (idx + i < n) out[idx + i] = run;
        run += v[i];
    }
    if (threadIdx.x == SCAN_THREADS - 1) {
        if (tile_sums) tile_sums[blockIdx.x] = run;
        if (total_out) *total_out = run;
    }
}

// Exclusive scan of a short array by one block: tiles of SCAN_TILE in order,
// each offset by the running total of the ones before (in place allowed).
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_block(const int* in, int* out, long n,
                                                             int* total_out)
{
    __shared__ int wsum[SCAN_THREADS / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int carry = 0;
    for (long t0 = 0; t0 < n; t0 += SCAN_TILE) {
        const long idx = t0 + (long)threadIdx.x * SCAN_ITEMS;
        int v[SCAN_ITEMS];
        int t = 0;
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; i++) {
            v[i] = (idx + i < n) ? in[idx + i] : 0;
            t += v[i];
        }
        const int incl = warp_incl_scan(t);
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const int s = wsum[lane];
            const int si = warp_incl_scan(s);
            wsum[lane] = si;
        }
        __syncthreads();
        int run = carry + incl - t + (warp ? wsum[warp - 1] : 0);
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; i++) {
            if (idx + i < n) out[idx + i] = run;
            run += v[i];
        }
        carry += wsum[31];
        __syncthreads();   // wsum reused by the next tile
    }
    if (total_out && threadIdx.x == 0) *total_out = carry;
}

// offsets[k] = the first position of sorted[0, N) holding a key >= k, for
// k <= nkeys: the start of each key's run (offsets[nkeys] = N).
__global__ void k_key_bounds(const int* __restrict__ sorted, int N, int nkeys,
                             int* __restrict__ offsets)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nkeys) return;
    int lo = 0, hi = N;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (sorted[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    offsets[k] = lo;
}

__global__ void k_scan_add(int* out, long n, const int* __restrict__ tile_offs, int ntiles,
                           int* total_out)
{
    const int add = tile_offs[blockIdx.x];
    const long base = (long)blockIdx.x * SCAN_TILE;
    for (int i = threadIdx.x; i < SCAN_TILE; i += blockDim.x) {
        const long j = base + i;
        if (j < n) out[j] += add;
    }
    if (total_out && blockIdx.x == 0 && threadIdx.x == 0) *total_out = tile_offs[ntiles];
}

__global__ void k_radix_hist(const int* __restrict__ keys, int N, int shift,
                             int* __restrict__ hist, int ntiles)
{
    __shared__ int cnt[RADIX];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const long base = (long)blockIdx.x * SORT_TILE;
    for (int r = 0; r < SORT_ROUNDS; r++) {
        const long i = base + r * SORT_THREADS + threadIdx.x;
        if (i < N) atomicAdd(&cnt[(keys[i] >> shift) & (RADIX - 1)], 1);
    }
    __syncthreads();
    hist[(long)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(SORT_THREADS) k_radix_scatter(
    const int* __restrict__ kin, const int* __restrict__ vin, int N, int shift,
    const int* __restrict__ hist, int ntiles, int* __restrict__ kout, int* __restrict__ vout)
{
    __shared__ int run[RADIX];
    __shared__ int wc[SORT_WARPS][RADIX];
    __shared__ int tile_base[RADIX];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    run[t] = 0;
    tile_base[t] = hist[(long)t * ntiles + blockIdx.x];
    const unsigned lt = (1u << lane) - 1u;
    const long base = (long)blockIdx.x * SORT_TILE;
    for (int r = 0; r < SORT_ROUNDS; r++) {
#pragma unroll
        for (int w = 0; w < SORT_WARPS; w++) wc[w][t] = 0;
        __syncthreads();
        const long i = base + r * SORT_THREADS + t;
        const bool valid = i < N;
        const int key = valid ? kin[i] : 0;
        const int d = valid ? ((key >> shift) & (RADIX - 1)) : RADIX;   // RADIX: no item
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt);
        if (valid && rank == 0) wc[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int before = run[d] + rank;
            for (int w = 0; w < warp; w++) before += wc[w][d];
            const int dest = tile_base[d] + before;
            kout[dest] = key;
            vout[dest] = vin ? vin[i] : (int)i;
        }
        __syncthreads();
        int s = 0;
#pragma unroll
        for (int w = 0; w < SORT_WARPS; w++) s += wc[w][t];
        run[t] += s;
        __syncthreads();
    }
}

__global__ void k_iota(int* out, int N)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) out[i] = (int)i;
}

int radix_passes(int nkeys)
{
    int bits = 0;
    while (bits < 31 && (1L << bits) < (long)nkeys) bits++;
    return (bits + RADIX_BITS - 1) / RADIX_BITS;
}

}  // namespace

size_t scan_scratch_bytes(long n)
{
    const long nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (n <= SCAN_BLOCK_MAX) return 0;
    return align_up(sizeof(int) * (nt + 1)) + scan_scratch_bytes(nt);
}

int exclusive_scan(const int* in, int* out, long n, bool write_total, void* scratch,
                   cudaStream_t st, int* launches)
{
    if (n <= 0) {
        if (write_total) SE_CUDA(cudaMemsetAsync(out, 0, sizeof(int), st));
        return SE_OK;
    }
    const long nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (n <= SCAN_BLOCK_MAX) {   // one block, one launch
        k_scan_block<<<1, SCAN_THREADS, 0, st>>>(in, out, n, write_total ? out + n : nullptr);
        SE_CUDA(cudaGetLastError());
        if (launches) (*launches)++;
        return SE_OK;
    }
    int* sums = static_cast<int*>(scratch);
    void* rest = static_cast<char*>(scratch) + align_up(sizeof(int) * (nt + 1));
    k_scan_tile<<<(unsigned)nt, SCAN_THREADS, 0, st>>>(in, out, n, sums, nullptr);
    SE_CUDA(cudaGetLastError());
    if (launches) (*launches)++;
    SE_TRY(exclusive_scan(sums, sums, nt, true, rest, st, launches));
    k_scan_add<<<(unsigned)nt, 256, 0, st>>>(out, n, sums, (int)nt, write_total ? out + n : nullptr);
    SE_CUDA(cudaGetLastError());
    if (launches) (*launches)++;
    return SE_OK;
}

size_t sort_scratch_bytes(int N, int nkeys)
{
    const long ntiles = (N + SORT_TILE - 1) / SORT_TILE;
    const long hist = (long)RADIX * (ntiles > 0 ? ntiles : 1);
    size_t b = 0;
    b += 4 * align_up(sizeof(int) * (size_t)(N > 0 ? N : 1));          // keys/vals ping-pong
    b += align_up(sizeof(int) * (size_t)(N > 0 ? N : 1));              // sorted keys if not wanted
    b += align_up(sizeof(int) * (size_t)(hist + 1));
    b += align_up(scan_scratch_bytes(hist));
    return b;
}

int stable_sort(const int* keys, const int* vals_in, int N, int nkeys, int* perm,
                int* sorted_keys, int* offsets, void* scratch, size_t scratch_bytes,
                cudaStream_t st, int* launches)
{
    if (N < 0 || nkeys < 1) return SE_ERR_INVALID;
    if (scratch_bytes < sort_scratch_bytes(N, nkeys)) return SE_ERR_INVALID;
    char* p = static_cast<char*>(scratch);
    const size_t nb = align_up(sizeof(int) * (size_t)(N > 0 ? N : 1));
    int* kA = reinterpret_cast<int*>(p); p += nb;
    int* vA = reinterpret_cast<int*>(p); p += nb;
    int* kB = reinterpret_cast<int*>(p); p += nb;
    int* vB = reinterpret_cast<int*>(p); p += nb;
    int* kS = reinterpret_cast<int*>(p); p += nb;
    const long ntiles = (N + SORT_TILE - 1) / SORT_TILE;
    const long nhist = (long)RADIX * (ntiles > 0 ? ntiles : 1);
    int* hist = reinterpret_cast<int*>(p); p += align_up(sizeof(int) * (size_t)(nhist + 1));
    void* sscr = p;
    int* kfinal = sorted_keys ? sorted_keys : kS;

    // the start of every key's run, from the sorted keys
    auto bounds = [&](const int* sorted) -> int {
        if (!offsets) return SE_OK;
        k_key_bounds<<<ceil_div((long)nkeys + 1, 256), 256, 0, st>>>(sorted, N, nkeys, offsets);
        SE_CUDA(cudaGetLastError());
        if (launches) (*launches)++;
        return SE_OK;
    };
    if (N == 0) return bounds(keys);
    const int passes = radix_passes(nkeys);
    if (passes == 0) {   // a single key: the identity permutation
        k_iota<<<ceil_div(N, 256), 256, 0, st>>>(perm, N);
        SE_CUDA(cudaGetLastError());
        if (launches) (*launches)++;
        if (sorted_keys) SE_CUDA(cudaMemcpyAsync(sorted_keys, keys, sizeof(int) * N,
                                                 cudaMemcpyDeviceToDevice, st));
        return bounds(keys);
    }
    const int* kin = keys;
    const int* vin = vals_in;
    for (int pass = 0; pass < passes; pass++) {
        const bool last = pass == passes - 1;
        int* kout = last ? kfinal : ((pass & 1) ? kB : kA);
        int* vout = last ? perm : ((pass & 1) ? vB : vA);
        const int shift = pass * RADIX_BITS;
        k_radix_hist<<<(unsigned)ntiles, RADIX, 0, st>>>(kin, N, shift, hist, (int)ntiles);
        SE_CUDA(cudaGetLastError());
        SE_TRY(exclusive_scan(hist, hist, nhist, false, sscr, st, launches));
        k_radix_scatter<<<(unsigned)ntiles, SORT_THREADS, 0, st>>>(kin, vin, N, shift, hist,
                                                                   (int)ntiles, kout, vout);
        SE_CUDA(cudaGetLastError());
        if (launches) (*launches) += 2;
        kin = kout;
        vin = vout;
    }
    return bounds(kfinal);
}

}  // namespace se

extern "C" size_t se_sort_scratch_bytes(int N, int nkeys)
{
    return se::sort_scratch_bytes(N, nkeys);
}

extern "C" int se_counting_sort(const int* keys, int N, int nkeys, int* perm, int* offsets,
                                void* scratch, size_t scratch_bytes, void* stream)
{
    return se::stable_sort(keys, nullptr, N, nkeys, perm, nullptr, offsets, scratch,
                           scratch_bytes, se::as_stream(stream), nullptr);
}
