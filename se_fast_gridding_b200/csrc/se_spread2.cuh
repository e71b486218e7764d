// se_spread2.cuh -- the spread (SE_FGG_grid, SE_fgg.c:3866-4028) with the
// periodic fold (SE_FGG_wrap_fcn, SE_fgg.c:327-352) fused, for the systems
// whose grid is cut into whole 16^3 tiles (M a multiple of 16, M >= 32) and
// whose stencil fits two tiles (P <= 16).  Included inside namespace se by
// se_solve.cu after se_spread.cuh (whose bin-range helpers it uses).
//
// Factor rows aligned to tiles.  k_factors writes, per particle and axis, a
// 32-entry row R[j] = f[j - s] (zero outside the stencil), where s = g mod 16
// is the stencil's start inside its home tile g / 16.  A stencil covers at
// most the home tile and the next one (periodically), and the row of tile
// home + h is R[16h .. 16h + 15]: one aligned 64-byte copy, no wrap logic.
//
// One CTA of 4 warps owns one 16^3 tile; warp w = 2 wy + wz owns the
// 16 x 8 x 8 block of y in 8 wy + [0, 8) and z in 8 wz + [0, 8), and the
// warps run independently, with no CTA barrier.  A warp lists the bin
// segments whose particles may reach its block (the tile's 16 x cells, its
// own 8 y and 8 z: at most 5 x 4 x 2 segments), walks their candidates in
// order, keeps the particles whose stencil meets the block and sorts them
// into three x classes -- the particle's x row in the tile meets both 8-cell
// halves, the low half only or the high half only -- one list ring each.
// Whenever a class holds a group (one particle per lane) the warp streams it
// through two shared-memory stages that cp.async fills from the factor rows
// while the warp works on the other: the x tile row (of a one-half class,
// that half), the warp's 8 y and 8 z entries and the charge.  Each lane adds
// px[x] * (q py[y] pz[z]) into the 16 x 2 cells of its (y, z) and
// (y, z + 1), or the 8 x 2 of the class's half: a one-half group costs half
// the FMAs of a full one, and a particle is a one-half particle in about
// half of the tiles it meets at P = 16 (more at smaller P).  Every cell
// belongs to one lane of one CTA: no atomics and a fixed order of summation
// (the groups' order, which depends only on the block's candidate list).
// FP32: packed FP32 pair FMAs on the cells, and after every 512 of the
// warp's particles the FP32 sums are added into the FP64 grid in place (the
// first time stored), which the lane alone reads and writes.
//
// Crowded tiles are split.  Each warp's candidate list is cut into parts of
// at most S2_CAP candidates; k_tile_parts counts the candidates of each
// tile's most crowded block and scans the part counts, and k_spread2 runs
// one CTA per part, whose warps take part s of their own lists.  Part 0
// writes the tile into the grid as above; part s >= 1 writes its sums into
// slab slot (extra parts of the tiles before it) + s - 1, 16^3 FP64 cells;
// the part that finishes last (a per-tile counter) adds the slabs into the
// grid in the order s = 1, 2, ...  A tile's parts and their sums depend only
// on its own candidates, so results stay deterministic and a batched
// system's grid equals its single solve's.  Uniform inputs at the
// configurations' densities have far fewer than S2_CAP candidates per block
// and are never split.

#ifndef SE_S2_CAP
#define SE_S2_CAP 8192
#endif
#ifndef SE_S2_UNROLL
#define SE_S2_UNROLL 16
#endif
constexpr int S2_CAP = SE_S2_CAP;   // candidates per part of a warp's list
constexpr int S2_WARPS = 4;   // warp blocks per tile
// warps per CTA: a tile's four warp blocks run as S2_WARPS / S2_CTA_WARPS
// CTAs (the warps are independent), so that the SMs share out the blocks
// more evenly (two CTAs of 2 warps per tile against one of 4: C2 spread
// 0.135 -> 0.128 ms, C3 2.33 -> 2.26 ms, C5 12.7 -> 11.6 ms)
#ifndef SE_S2_CTA_WARPS
#define SE_S2_CTA_WARPS 2
#endif
constexpr int S2_CTA_WARPS = SE_S2_CTA_WARPS;
static_assert(S2_WARPS % S2_CTA_WARPS == 0, "a tile's warp blocks split evenly into CTAs");
// grids of at least S2_ONE_WARP_TILES tiles (the 5-CTA build) run one warp
// per CTA instead (the M = 512 clustered spread 11.48 -> 11.13 ms; smaller
// grids measured better with two)
#ifndef SE_S2_ONE_WARP_TILES
#define SE_S2_ONE_WARP_TILES 32768
#endif
constexpr int S2_ONE_WARP_TILES = SE_S2_ONE_WARP_TILES;
constexpr int S2_LIST = 64;    // per-class list ring: >= group - 1 + 32
constexpr int S2_SEGS = 64;    // bin segments reaching a warp's block: <= 5 x 4 x 2 for P <= 16
constexpr int S2_FOLD = 512;   // FP32 partial sums cover this many of a warp's particles
// x classes of a particle in a tile: its x row meets both 8-cell halves,
// the low half only, the high half only
constexpr int S2_CLASSES = 3;
constexpr int S2_UNROLL = SE_S2_UNROLL;   // particles per unrolled pass of a group
// FP32 CTAs per SM the kernel is compiled for: 5 (96 registers) where the
// tiles outnumber 4 CTAs per SM, 4 (128 registers) where all of them are
// resident at once either way; FP64: 3
constexpr int S2_BLOCKS_MANY = 5, S2_BLOCKS_FEW = 4, S2_BLOCKS_FP64 = 3;

// particles a warp stages at once: one per lane (FP32), half a warp (FP64)
template <typename Acc>
constexpr int s2_group() { return sizeof(Acc) == 4 ? 32 : 16; }

template <typename Acc>
struct Spread2Stage {
    Acc px[s2_group<Acc>()][16];
    Acc pz[s2_group<Acc>()][8];
    Acc py[s2_group<Acc>()][8];
    double q[s2_group<Acc>()];
};

template <typename Acc, int CW>
struct Spread2Smem {
    Spread2Stage<Acc> stage[CW][2];
    int2 list[CW][S2_CLASSES][S2_LIST];   // (particle, packed grid index)
    int seg_beg[CW][S2_SEGS];
    int seg_pre[CW][S2_SEGS];
};

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The 32 cells of one lane: 16 x for z and for z + 1.
template <typename Acc>
struct Spread2Accum;

template <>
struct Spread2Accum<float> {
    float2 a[8], b[8];   // packed x pairs for z and z + 1
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = b[m] = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void add(const float* px, float c0, float c1)
    {
        const float2 k0 = f32x2(c0, c0), k1 = f32x2(c1, c1);
        const float4* p4 = reinterpret_cast<const float4*>(px);
#pragma unroll
        for (int m = 0; m < 4; m++) {
            float2 lo, hi;
            f32x2_split(p4[m], lo, hi);
            a[2 * m] = ffma2(lo, k0, a[2 * m]);
            a[2 * m + 1] = ffma2(hi, k0, a[2 * m + 1]);
            b[2 * m] = ffma2(lo, k1, b[2 * m]);
            b[2 * m + 1] = ffma2(hi, k1, b[2 * m + 1]);
        }
    }
    // x in [8 H, 8 H + 8) only (the row is zero on the other half)
    template <int H>
    __device__ __forceinline__ void add_half(const float* px, float c0, float c1)
    {
        const float2 k0 = f32x2(c0, c0), k1 = f32x2(c1, c1);
        const float4* p4 = reinterpret_cast<const float4*>(px);
#pragma unroll
        for (int m = 2 * H; m < 2 * H + 2; m++) {
            float2 lo, hi;
            f32x2_split(p4[m], lo, hi);
            a[2 * m] = ffma2(lo, k0, a[2 * m]);
            a[2 * m + 1] = ffma2(hi, k0, a[2 * m + 1]);
            b[2 * m] = ffma2(lo, k1, b[2 * m]);
            b[2 * m + 1] = ffma2(hi, k1, b[2 * m + 1]);
        }
    }
    // cell (x, z + zz) at cell0 + x * plane + zz: the FP64 grid value plus
    // this lane's FP32 partial sums (or the sums alone the first time)
    __device__ __forceinline__ void fold(double* cell0, long long plane, bool first)
    {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            double2 old[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
                old[k] = first ? make_double2(0.0, 0.0)
                               : *reinterpret_cast<const double2*>(cell0 + (8 * h + k) * plane);
#pragma unroll
            for (int k = 0; k < 8; k += 2) {
                const int m = 4 * h + k / 2;
                const float2 u = a[m], v = b[m];
                *reinterpret_cast<double2*>(cell0 + (8 * h + k) * plane) =
                    make_double2(old[k].x + (double)u.x, old[k].y + (double)v.x);
                *reinterpret_cast<double2*>(cell0 + (8 * h + k + 1) * plane) =
                    make_double2(old[k + 1].x + (double)u.y, old[k + 1].y + (double)v.y);
                a[m] = b[m] = make_float2(0.f, 0.f);
            }
        }
    }
};

template <>
struct Spread2Accum<double> {
    double a[16], b[16];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int x = 0; x < 16; x++) a[x] = b[x] = 0.0;
    }
    __device__ __forceinline__ void add(const double* px, double c0, double c1)
    {
        const double2* p2 = reinterpret_cast<const double2*>(px);
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const double2 w = p2[m];
            a[2 * m] = fma(w.x, c0, a[2 * m]);
            a[2 * m + 1] = fma(w.y, c0, a[2 * m + 1]);
            b[2 * m] = fma(w.x, c1, b[2 * m]);
            b[2 * m + 1] = fma(w.y, c1, b[2 * m + 1]);
        }
    }
    template <int H>
    __device__ __forceinline__ void add_half(const double* px, double c0, double c1)
    {
        const double2* p2 = reinterpret_cast<const double2*>(px);
#pragma unroll
        for (int m = 4 * H; m < 4 * H + 4; m++) {
            const double2 w = p2[m];
            a[2 * m] = fma(w.x, c0, a[2 * m]);
            a[2 * m + 1] = fma(w.y, c0, a[2 * m + 1]);
            b[2 * m] = fma(w.x, c1, b[2 * m]);
            b[2 * m + 1] = fma(w.y, c1, b[2 * m + 1]);
        }
    }
    __device__ __forceinline__ void store(double* cell0, long long plane) const
    {
#pragma unroll
        for (int x = 0; x < 16; x++)
            *reinterpret_cast<double2*>(cell0 + x * plane) = make_double2(a[x], b[x]);
    }
};

// Half h in {0, 1} of the home tile t0 = g / 16 that is tile ti, or -1 when
// the stencil [g, g + P) misses tile ti (nt tiles per axis, periodic).
__device__ __forceinline__ int tile_half(int g, int ti, int nt, int P)
{
    int h = ti - (g >> 4);
    if (h < 0) h += nt;
    if (h == 0) return 0;
    return (h == 1 && (g & 15) + P > 16) ? 1 : -1;
}

// The bins whose particles may reach block (wy, wz) of a tile at corner
// (x0, y0, z0) -- x: the tile's 16 cells, y and z: the block's 8 -- as
// segments (x bin, y bin, z run) numbered x-major; a z run is a contiguous
// range of bins, so a segment is a contiguous range of the sorted particles.
struct BlockBins {
    BinRanges rx, ry, rz;
    int nx, ny;
    __device__ __forceinline__ BlockBins(const SysDev& S, int x0, int y0, int z0)
        : rx(bins_reaching(x0, 16, S.M, S.P, S.nf[0])),
          ry(bins_reaching(y0, 8, S.M, S.P, S.nf[1])),
          rz(bins_reaching(z0, 8, S.M, S.P, S.nf[2])),
          nx(range_count(rx)), ny(range_count(ry))
    {
    }
    __device__ __forceinline__ int segments() const { return nx * ny * 2; }
    // the particles [beg, beg + len) of segment u
    __device__ __forceinline__ void segment(const SysDev& S, const int* __restrict__ boff, int u,
                                            int& beg, int& len) const
    {
        const int zr = u & 1, iy = (u >> 1) % ny, ix = (u >> 1) / ny;
        const int bz0 = zr ? rz.b0 : rz.a0, bz1 = zr ? rz.b1 : rz.a1;
        beg = 0;
        len = 0;
        if (bz0 <= bz1) {
            const int kb = S.bin_base + (range_at(rx, ix) * S.nf[1] + range_at(ry, iy)) * S.nf[2];
            beg = boff[kb + bz0];
            len = boff[kb + bz1 + 1] - beg;
        }
    }
};

// The number of candidates (the particles of the bin segments that reach
// it) of warp block w of tile lt of system S; every lane gets it.
__device__ __forceinline__ int block_candidates(const SysDev& S, int lt, int w,
                                                const int* __restrict__ boff, int lane)
{
    const int nt = S.nt[0];
    const int tix = lt / (nt * nt), tiy = (lt / nt) % nt, tiz = lt % nt;
    const BlockBins B(S, tix * 16, tiy * 16 + 8 * (w >> 1), tiz * 16 + 8 * (w & 1));
    int sum = 0;
    for (int u = lane; u < B.segments(); u += 32) {
        int beg, len;
        B.segment(S, boff, u, beg, len);
        sum += len;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    return sum;
}

// Parts per tile (one warp per warp block, two tiles per CTA:
// max(1, ceil(candidates of the most crowded block / S2_CAP)) for the
// k_spread2 systems, 1 for the others), then, in the block that finishes
// last, their exclusive scan in place: parts[t] = the first part of tile t,
// parts[ntiles] = the number of parts, and part_tile[s] = the tile of part s.  More parts than the launch bound
// (which no input reaches: a bin is a candidate of at most two tiles per
// axis) set bit 2 of err.  The block counter is left at zero for the next
// launch.
constexpr int TP_WARPS = 8;
constexpr int TP_TILES = TP_WARPS / S2_WARPS;   // tiles per CTA

__global__ void __launch_bounds__(TP_WARPS * 32) k_tile_parts(
    const SysDev* __restrict__ sys, const int* __restrict__ tile_prefix, int nsys, int ntiles,
    const int* __restrict__ boff, int* parts, unsigned* counter, int bound, int* err,
    int* __restrict__ part_tile)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * TP_TILES + warp / S2_WARPS, wb = warp % S2_WARPS;
    __shared__ int cand[TP_WARPS];
    int c = 0;
    if (tile < ntiles) {
        const SysDev& S = sys[find_sys(tile_prefix, nsys, tile)];
        if (S.path & PATH_TILE_SPREAD) c = block_candidates(S, tile - S.tile_base, wb, boff, lane);
    }
    if (lane == 0) cand[warp] = c;
    __syncthreads();
    if (wb == 0 && lane == 0 && tile < ntiles) {
        int most = 0;
#pragma unroll
        for (int k = 0; k < S2_WARPS; k++) most = max(most, cand[warp + k]);
        parts[tile] = max(1, (most + S2_CAP - 1) / S2_CAP);
    }
    __shared__ int last;
    __shared__ int wsum[TP_WARPS];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    int carry = 0;
    for (int t0 = 0; t0 < ntiles; t0 += TP_WARPS * 32 * 4) {
        const int idx = t0 + threadIdx.x * 4;
        int v[4], sum = 0;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            v[i] = idx + i < ntiles ? __ldcg(parts + idx + i) : 0;
            sum += v[i];
        }
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        int before = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < TP_WARPS; w++) {
            before += w < warp ? wsum[w] : 0;
            tot += wsum[w];
        }
        int run = carry + before + incl - sum;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (idx + i < ntiles) parts[idx + i] = run;
            run += v[i];
        }
        carry += tot;
        __syncthreads();   // wsum is reused
    }
    if (threadIdx.x == 0) {
        parts[ntiles] = carry;
        if (carry > bound) atomicOr(err, 2);
        *counter = 0u;
    }
    // every part's tile, for k_spread2 (the first `bound` parts)
    __syncthreads();
    for (int t = threadIdx.x; t < ntiles; t += blockDim.x) {
        const int a = __ldcg(parts + t), b = min(__ldcg(parts + t + 1), bound);
        for (int s = a; s < b; s++) part_tile[s] = t;
    }
}

// CW warps per CTA (S2_WARPS / CW CTAs per part of a tile)
template <typename Acc, int BLOCKS, int CW = S2_CTA_WARPS>
__global__ void __launch_bounds__(CW * 32, BLOCKS * (S2_WARPS / CW)) k_spread2(
    const SysDev* __restrict__ sys, const int* __restrict__ tile_sys,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const Acc* __restrict__ rows, const int* __restrict__ boff, double* __restrict__ grid,
    const int* __restrict__ tile_parts, const int* __restrict__ part_tile, int ntiles,
    int* __restrict__ tile_done, double* __restrict__ slab, int slab_slots,
    int* __restrict__ err)
{
    constexpr bool FOLD = sizeof(Acc) == 4;
    constexpr int G = s2_group<Acc>();
    constexpr int V = 16 / sizeof(Acc);   // entries per 16-byte copy
    constexpr int S2_CTA_SPLIT = S2_WARPS / CW, S2_THREADS = CW * 32;
    __shared__ __align__(16) Spread2Smem<Acc, CW> sm;
    __shared__ int folds;   // this CTA finished its tile's parts last

    // ---- the part this CTA sums and its tile (k_tile_parts' part_tile; warp
    // blocks sub CW + [0, CW) of it), and the tile's system
    const int item = blockIdx.x / S2_CTA_SPLIT, sub = blockIdx.x % S2_CTA_SPLIT;
    const int nall = tile_parts[ntiles];
    const int tile = part_tile[item];   // (the grid holds at most `bound` parts)
    if (item >= nall) return;
    if ((unsigned)tile >= (unsigned)ntiles) {   // cannot happen: flagged, nothing summed
        if (threadIdx.x == 0) atomicOr(err, 2);
        return;
    }
    const int first = tile_parts[tile];
    const int ipart = item - first;
    const int nparts = tile_parts[tile + 1] - first;
    const SysDev& S = sys[tile_sys[tile]];
    if (!(S.path & PATH_TILE_SPREAD)) return;   // k_spread covers this system
    const int slot0 = tile_parts[tile] - tile;   // slab slot of part 1
    if (ipart > 0 && slot0 + ipart - 1 >= slab_slots) {   // cannot happen: see k_tile_parts
        if (threadIdx.x == 0) atomicOr(err, 2);
        return;
    }
    const int nt = S.nt[0], P = S.P, M = S.M;
    const int lt = tile - S.tile_base;
    const int tix = lt / (nt * nt), tiy = (lt / nt) % nt, tiz = lt % nt;
    const int x0 = tix * 16, y0 = tiy * 16, z0 = tiz * 16;
    const int t = threadIdx.x, lw = t >> 5, lane = t & 31;
    const int warp = sub * CW + lw;   // the warp block of the tile
    const int wy = warp >> 1, wz = warp & 1;
    const int ly = lane >> 2, lz = (lane & 3) * 2;
    const unsigned ybits = 0xFFu << (8 * wy), zbits = 0xFFu << (8 * wz);

    // ---- the bin segments reaching this warp's block (at most 5 x 4 x 2) and
    // their prefix: the warp's own candidate list, in segment order
    const BlockBins B(S, x0, y0 + 8 * wy, z0 + 8 * wz);
    int nseg = B.segments();
    if (nseg > S2_SEGS) {   // cannot happen for M >= 32 and P <= 16: flagged, the block sums nothing
        if (lane == 0) atomicOr(err, 2);
        nseg = 0;
    }
    int* seg_beg = sm.seg_beg[lw];
    int* seg_pre = sm.seg_pre[lw];
    int total = 0;
    for (int u0 = 0; u0 < nseg; u0 += 32) {
        const int u = u0 + lane;
        int beg = 0, len = 0;
        if (u < nseg) B.segment(S, boff, u, beg, len);
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (u < nseg) {
            seg_beg[u] = beg;
            seg_pre[u] = total + incl - len;
        }
        total += __shfl_sync(0xffffffffu, incl, 31);
    }
    __syncwarp();   // the warps are independent from here on

    const unsigned pmask = (1u << P) - 1u;   // P <= 16
    const unsigned lanes_before = (1u << lane) - 1u;
    double* gs = grid + S.grid_off;
    const long long gplane = (long long)M * M;
    // part 0 sums into the grid, the others into their slab slot
    // (cells [x][y][z] of the tile, 16^3)
    const long long plane = ipart == 0 ? gplane : 256;
    double* cell0 =
        ipart == 0 ? gs + (long long)x0 * gplane + (long long)(y0 + 8 * wy + ly) * M + z0 + 8 * wz + lz
                  : slab + (long long)(slot0 + ipart - 1) * 4096 + (8 * wy + ly) * 16 + 8 * wz + lz;
    // this part's candidates: [cbeg, cend) of the warp's list
    const int cbeg = ipart * S2_CAP, cend = min(total, cbeg + S2_CAP);

    Spread2Accum<Acc> acc;
    acc.zero();
    // one ring per x class: byte c of cnt holds the entries of class c
    // listed and not yet staged (< 64), byte c of ring the slot of the first
    unsigned cnt = 0u, ring = 0u;
    // a class holds a group when its count has a bit of value >= G
    constexpr unsigned FULL = (G == 32 ? 0x20u : 0x30u) * 0x010101u;
    int cpos = cbeg, buf = 0, pending = 0, pcls = 0, since_fold = 0;
    int seg = 0;   // the segment holding candidate cpos
    while (seg + 1 < nseg && seg_pre[seg + 1] <= cpos) seg++;
    bool written = false;
    for (;;) {
        // ---- list until some class holds a group (or every remaining
        // candidate is listed), each class in candidate order
        while (!(cnt & FULL) && cpos < cend) {
            const int pos = cpos + lane;
            int part = -1, pk = 0, cls = -1, sl = seg;   // this lane's segment, found forward
            if (pos < cend) {
                while (sl + 1 < nseg && seg_pre[sl + 1] <= pos) sl++;
                part = seg_beg[sl] + (pos - seg_pre[sl]);
                pk = sg[part];
                // the stencil's cells in this tile, as 16-bit masks per axis
                const int gx = g_of(pk, 0), gy = g_of(pk, 1), gz = g_of(pk, 2);
                const int hx = tile_half(gx, tix, nt, P);
                const int hy = tile_half(gy, tiy, nt, P), hz = tile_half(gz, tiz, nt, P);
                const unsigned xm = ((pmask << (gx & 15)) >> (16 * max(hx, 0))) & 0xFFFFu;
                const bool meets = hx >= 0 && hy >= 0 && hz >= 0 &&
                                   ((((pmask << (gy & 15)) >> (16 * hy)) & 0xFFFFu) & ybits) &&
                                   ((((pmask << (gz & 15)) >> (16 * hz)) & 0xFFFFu) & zbits);
                if (meets) cls = (xm & 0xFFu) ? ((xm & 0xFF00u) ? 0 : 1) : 2;
            }
            const unsigned k0 = __ballot_sync(0xffffffffu, cls == 0);
            const unsigned k1 = __ballot_sync(0xffffffffu, cls == 1);
            const unsigned k2 = __ballot_sync(0xffffffffu, cls == 2);
            if (cls >= 0) {
                const unsigned kc = cls == 0 ? k0 : (cls == 1 ? k1 : k2);
                const int sh = 8 * cls;
                sm.list[lw][cls][((ring >> sh) + (cnt >> sh) + __popc(kc & lanes_before)) &
                                   (S2_LIST - 1)] = make_int2(part, pk);
            }
            cnt += __popc(k0) | (__popc(k1) << 8) | (__popc(k2) << 16);
            cpos += 32;
            seg = __reduce_max_sync(0xffffffffu, sl);
        }
        __syncwarp();   // list entries visible to the warp
        // ---- the class to stage: a full group if some class has one (the
        // first such class), else the first class with entries left
        const unsigned pick = (cnt & FULL) ? (cnt & FULL) : cnt;
        const int cls = pick ? (__ffs(pick) - 1) >> 3 : 0;
        const int sh = 8 * cls;
        const int avail = (cnt >> sh) & 0xFF;
        const int head = (ring >> sh) & (S2_LIST - 1);
        const int2* list = sm.list[lw][cls];
        // ---- stage the next group of the class: lane l < n copies its
        // particle head + l (of a one-half class, that half of the x row)
        const int n = min(G, avail);
        if (n > 0) {
            Spread2Stage<Acc>& st = sm.stage[lw][buf];
            if (lane < n) {
                const int2 e = list[(head + lane) & (S2_LIST - 1)];
                const int hx = tile_half(g_of(e.y, 0), tix, nt, P);
                const int hy = tile_half(g_of(e.y, 1), tiy, nt, P);
                const int hz = tile_half(g_of(e.y, 2), tiz, nt, P);
                const Acc* r = rows + (long long)e.x * 96;
                if (cls == 0) {
#pragma unroll
                    for (int k = 0; k < 16; k += V) cp_async16(&st.px[lane][k], r + 16 * hx + k);
                } else {
                    const int o = 8 * (cls - 1);
#pragma unroll
                    for (int k = 0; k < 8; k += V) cp_async16(&st.px[lane][o + k], r + 16 * hx + o + k);
                }
#pragma unroll
                for (int k = 0; k < 8; k += V) {
                    cp_async16(&st.py[lane][k], r + 32 + 16 * hy + 8 * wy + k);
                    cp_async16(&st.pz[lane][k], r + 64 + 16 * hz + 8 * wz + k);
                }
                cp_async8(&st.q[lane], &srec[e.x].w);
            } else if (lane < G) {   // a short group: zero rows up to G (FP64: 16),
                                     // so every group sums G rows
#pragma unroll
                for (int k = 0; k < 16; k++) st.px[lane][k] = Acc(0);
#pragma unroll
                for (int k = 0; k < 8; k++) st.py[lane][k] = st.pz[lane][k] = Acc(0);
                st.q[lane] = 0.0;
            }
            cp_async_commit();
            cnt -= (unsigned)n << sh;
            ring = (ring & ~(0xFFu << sh)) | ((unsigned)((head + n) & (S2_LIST - 1)) << sh);
        }
        __syncwarp();   // the staged entries are read before the list refills over them
        // ---- the previous group, while this one lands
        if (pending > 0) {
            if (n > 0) cp_async_wait<1>();
            else cp_async_wait<0>();
            __syncwarp();
            Spread2Stage<Acc>& st = sm.stage[lw][buf ^ 1];
            // lane i scales its particle's 8 y entries by the charge, once
            if (lane < pending) {
                const Acc qv = (Acc)st.q[lane];
#pragma unroll
                for (int k = 0; k < 8; k++) st.py[lane][k] = st.py[lane][k] * qv;
            }
            __syncwarp();
            // every group holds G rows (a short one padded with zeros, which
            // add exact zeros): one unrolled pass per class with constant
            // offsets; a one-half class touches the lane's 8 x 2 cells of its half
            if (pcls == 0) {
#pragma unroll S2_UNROLL
                for (int i = 0; i < G; i++) {
                    const Acc y = st.py[i][ly];
                    acc.add(st.px[i], y * st.pz[i][lz], y * st.pz[i][lz + 1]);
                }
            } else if (pcls == 1) {
#pragma unroll S2_UNROLL
                for (int i = 0; i < G; i++) {
                    const Acc y = st.py[i][ly];
                    acc.template add_half<0>(st.px[i], y * st.pz[i][lz], y * st.pz[i][lz + 1]);
                }
            } else {
#pragma unroll S2_UNROLL
                for (int i = 0; i < G; i++) {
                    const Acc y = st.py[i][ly];
                    acc.template add_half<1>(st.px[i], y * st.pz[i][lz], y * st.pz[i][lz + 1]);
                }
            }
            if constexpr (FOLD) {
                since_fold += pending;
                if (since_fold >= S2_FOLD) {
                    acc.fold(cell0, plane, !written);
                    written = true;
                    since_fold = 0;
                }
            }
            __syncwarp();   // the stage is read before it is refilled
        }
        if (n == 0) break;
        pending = n;
        pcls = cls;
        buf ^= 1;
    }

    // ---- the lane's cells
    if constexpr (FOLD) {
        if (since_fold > 0 || !written) acc.fold(cell0, plane, !written);
    } else {
        acc.store(cell0, plane);
    }

    // ---- a split tile: the part that finishes last adds the slabs into the
    // grid, in part order
    if (nparts > 1) {
        __threadfence();
        __syncthreads();
        if (t == 0) folds = atomicAdd(&tile_done[tile], 1) == nparts * S2_CTA_SPLIT - 1;
        __syncthreads();
        if (folds) {
            __threadfence();
            for (int c = t; c < 4096; c += S2_THREADS) {
                const int x = c >> 8, y = (c >> 4) & 15, z = c & 15;
                double* gp = gs + (long long)(x0 + x) * gplane + (long long)(y0 + y) * M + z0 + z;
                double v = __ldcg(gp);
                for (int k = 0; k < nparts - 1; k++)
                    v += __ldcg(slab + (long long)(slot0 + k) * 4096 + c);
                *gp = v;
            }
            if (t == 0) tile_done[tile] = 0;
        }
    }
}
