// se_binsort.cuh -- the particle sort of a solve in three kernels, for
// batches of at most BSORT_MAX_KEYS fine bins and BSORT_MAX_N particles.
// Included inside namespace se by se_solve.cu after particle_of.
//
// The result is the stable counting sort by bin key (ties in particle order)
// that the radix path in se_sort.cu computes -- the same permutation, bit for
// bit, since a stable order is unique -- with the preparation before it and
// the gather after it fused in:
//
//   k_bsort_count    one CTA per chunk of consecutive particles: bin keys and
//                    the chunk's key histogram, row H[chunk][key];
//   k_bsort_columns  per key, the exclusive prefix of H down the chunks (in
//                    place) and the key's total T[key];
//   k_bsort_scatter  per chunk: the bin offsets (exclusive scan of T; chunk 0
//                    stores them), plus the chunk's column of H gives the
//                    first slot of each key; the chunk's keys are staged in
//                    shared memory, one warp walks them in particle order,
//                    ranking equal keys by voting on the key bits, and then
//                    every thread stores its particles' sorted record, packed
//                    grid index and source index at their slots (the factor
//                    rows follow from these in k_factors, whose warps store
//                    whole rows of consecutive slots).
//
// SE_FGG_reorder_system (SE_fgg.c:5894-5932) orders particles the same way
// (by its qsort over bin index) for the same reason: bin-ordered stencils.

constexpr int BSORT_THREADS = 512;
constexpr int BSORT_MAX_KEYS = 8192;
constexpr int BSORT_MAX_N = 1 << 19;
constexpr int BSORT_MAX_CHUNKS = 296;
constexpr int BSORT_MIN_CHUNK = 256;

// Particles per chunk for ntot particles: at least BSORT_MIN_CHUNK, at most
// BSORT_MAX_CHUNKS chunks, a multiple of 32.
__host__ __device__ inline int bsort_chunk(int ntot)
{
    int c = (ntot + BSORT_MAX_CHUNKS - 1) / BSORT_MAX_CHUNKS;
    c = c < BSORT_MIN_CHUNK ? BSORT_MIN_CHUNK : c;
    return (c + 31) & ~31;
}

inline bool bsort_fits(int ntot, int nkeys)
{
    return ntot > 0 && ntot <= BSORT_MAX_N && nkeys >= 1 && nkeys <= BSORT_MAX_KEYS;
}

// H (BSORT_MAX_CHUNKS x nkeys) and T (nkeys)
inline size_t bsort_scratch_bytes(int nkeys)
{
    return sizeof(int) * ((size_t)BSORT_MAX_CHUNKS + 1) * (size_t)nkeys;
}

inline size_t bsort_scatter_smem(int ntot, int nkeys)
{
    return sizeof(int) * ((size_t)nkeys + (size_t)bsort_chunk(ntot));
}

__global__ void __launch_bounds__(BSORT_THREADS) k_bsort_count(
    const SysDev* __restrict__ sys, const int* __restrict__ part_prefix, int nsys, int ntot,
    const double* __restrict__ x, const double* __restrict__ q, int chunk, int nkeys,
    int* __restrict__ key, int* __restrict__ H, int* err)
{
    extern __shared__ int cnt[];
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    const int c0 = blockIdx.x * chunk, c1 = min(ntot, c0 + chunk);
    bool bad = false;
    for (int n = c0 + threadIdx.x; n < c1; n += blockDim.x) {
        const SysDev& S = sys[find_sys(part_prefix, nsys, n)];
        double4 r;
        int g, k;
        bad |= !particle_of(S, x, q, n, r, g, k);
        key[n] = k;
        atomicAdd(&cnt[k], 1);
    }
    if (bad) atomicOr(err, 1);
    __syncthreads();
    int* row = H + (long long)blockIdx.x * nkeys;
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) row[k] = cnt[k];
}

// 32 keys per CTA (one per lane); its 8 warps take consecutive runs of at
// most BSORT_COL_RUN chunks.
constexpr int BSORT_COL_WARPS = 8;
constexpr int BSORT_COL_RUN = (BSORT_MAX_CHUNKS + BSORT_COL_WARPS - 1) / BSORT_COL_WARPS;

__global__ void __launch_bounds__(BSORT_COL_WARPS * 32) k_bsort_columns(
    int* __restrict__ H, int nchunks, int nkeys, int* __restrict__ T)
{
    __shared__ int seg[BSORT_COL_WARPS][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = blockIdx.x * 32 + lane;
    const int per = (nchunks + BSORT_COL_WARPS - 1) / BSORT_COL_WARPS;
    const int r0 = min(nchunks, warp * per), r1 = min(nchunks, r0 + per);
    int v[BSORT_COL_RUN];
    int s = 0;
#pragma unroll
    for (int i = 0; i < BSORT_COL_RUN; i++) {
        v[i] = (k < nkeys && r0 + i < r1) ? H[(long long)(r0 + i) * nkeys + k] : 0;
        s += v[i];
    }
    seg[warp][lane] = s;
    __syncthreads();
    int run = 0, total = 0;
#pragma unroll
    for (int w = 0; w < BSORT_COL_WARPS; w++) {
        const int c = seg[w][lane];
        run += w < warp ? c : 0;
        total += c;
    }
    if (k >= nkeys) return;
#pragma unroll
    for (int i = 0; i < BSORT_COL_RUN; i++) {
        if (r0 + i < r1) H[(long long)(r0 + i) * nkeys + k] = run;
        run += v[i];
    }
    if (warp == 0) T[k] = total;
}

__global__ void __launch_bounds__(BSORT_THREADS, 3) k_bsort_scatter(
    const SysDev* __restrict__ sys, const int* __restrict__ part_prefix, int nsys, int ntot,
    const double* __restrict__ x, const double* __restrict__ q, int chunk, int nkeys,
    const int* __restrict__ key, const int* __restrict__ H, const int* __restrict__ T,
    int* __restrict__ boff, int* __restrict__ perm, double4* __restrict__ srec,
    int* __restrict__ sg, int* err)
{
    extern __shared__ int sm[];
    int* slot = sm;           // [nkeys]: the next slot of each key
    int* dst = sm + nkeys;    // [chunk]: each particle's key, then its slot
    __shared__ int wsum[BSORT_THREADS / 32];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int c0 = blockIdx.x * chunk, c1 = min(ntot, c0 + chunk);
    for (int n = c0 + t; n < c1; n += BSORT_THREADS) dst[n - c0] = key[n];

    // ---- bin offsets: exclusive scan of T, a contiguous run of keys per thread
    const int per = (nkeys + BSORT_THREADS - 1) / BSORT_THREADS;
    const int k0 = min(nkeys, t * per), k1 = min(nkeys, k0 + per);
    int mine = 0;
    for (int k = k0; k < k1; k++) mine += T[k];
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = 0;
#pragma unroll
    for (int w = 0; w < BSORT_THREADS / 32; w++) before += w < warp ? wsum[w] : 0;
    int run = before + incl - mine;
    const int* col = H + (long long)blockIdx.x * nkeys;
    for (int k = k0; k < k1; k++) {
        if (blockIdx.x == 0) boff[k] = run;
        slot[k] = run + col[k];
        run += T[k];
    }
    if (blockIdx.x == 0 && t == BSORT_THREADS - 1) boff[nkeys] = run;
    __syncthreads();

    // ---- ranks, in particle order, by one warp (keys replaced by slots).
    // Lanes holding equal keys: the lanes that agree with this one on every
    // key bit (one ballot per bit).
    if (warp == 0) {
        int nbits = 0;
        while ((1 << nbits) < nkeys) nbits++;
        const unsigned lt = (1u << lane) - 1u;
        for (int b = c0; b < c1; b += 32) {
            const int n = b + lane;
            const bool valid = n < c1;
            const int k = valid ? dst[n - c0] : 0;
            unsigned peers = __ballot_sync(0xffffffffu, valid);
            for (int i = 0; i < nbits; i++) {
                const bool bit = (k >> i) & 1;
                const unsigned m = __ballot_sync(0xffffffffu, bit);
                peers &= bit ? m : ~m;
            }
            const int leader = __ffs(peers) - 1;   // valid lanes: peers holds this lane
            int base = 0;
            if (valid && lane == leader) {
                base = slot[k];
                slot[k] = base + __popc(peers);
            }
            base = __shfl_sync(0xffffffffu, base, valid ? leader : lane);
            if (valid) dst[n - c0] = base + __popc(peers & lt);
            __syncwarp();
        }
    }
    __syncthreads();

    // ---- the sorted records, at the slots
    bool bad = false;
    for (int n = c0 + t; n < c1; n += BSORT_THREADS) {
        const int d = dst[n - c0];
        if (d < 0 || d >= ntot) {   // cannot happen with consistent counts
            bad = true;
            continue;
        }
        const SysDev& S = sys[find_sys(part_prefix, nsys, n)];
        double4 r;
        int g, k;
        particle_of(S, x, q, n, r, g, k);
        srec[d] = r;
        sg[d] = g;
        perm[d] = n;
    }
    if (bad) atomicOr(err, 4);
}
