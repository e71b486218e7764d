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
// 16 x 8 x 8 block of y in 8 wy + [0, 8) and z in 8 wz + [0, 8), and after
// the CTA has listed the bin segments that reach the tile the warps run
// independently, with no CTA barrier: each warp walks the candidates of the
// segments in order, keeps the particles whose stencil meets its block, and
// streams them in groups -- one particle per lane -- through two
// shared-memory stages that cp.async fills from the factor rows while the
// warp works on the other: the x tile row, the warp's 8 y and 8 z entries and
// the charge.  Each lane adds px[x] * (q py[y] pz[z]) into 16 x 2 cells (all
// 16 x of its (y, z) and (y, z + 1)).  Every cell belongs to one lane of one CTA: no atomics and a
// fixed order of summation (the particles' candidate order).  FP32:
// packed FP32 pair FMAs on the cells, and after every 512 of the warp's
// particles the FP32 sums are added into the FP64 grid in place (the first
// time stored), which the lane alone reads and writes.
//
// Crowded tiles are split.  A tile's candidate list (the particles of the
// bin segments that reach it, in bin order) is cut into parts of at most
// S2_CAP candidates; k_tile_parts counts each tile's candidates and scans the
// part counts, and k_spread2 runs one CTA per part.  Part 0 writes the tile
// into the grid as above; part s >= 1 writes its sums into slab slot
// (extra parts of the tiles before it) + s - 1, 16^3 FP64 cells; the part
// that finishes last (a per-tile counter) adds the slabs into the grid in
// the order s = 1, 2, ...  A tile's parts and their sums depend only on its
// own candidates, so results stay deterministic and a batched system's grid
// equals its single solve's.  Uniform inputs at the configurations' densities
// have far fewer than S2_CAP candidates per tile and are never split.

#ifndef SE_S2_CAP
#define SE_S2_CAP 8192
#endif
#ifndef SE_S2_MIN_BLOCKS
#define SE_S2_MIN_BLOCKS 5
#endif
#ifndef SE_S2_FULL_GROUP
#define SE_S2_FULL_GROUP 1
#endif
constexpr int S2_CAP = SE_S2_CAP;   // candidates per part of a tile
constexpr int S2_WARPS = 4;
constexpr int S2_THREADS = S2_WARPS * 32;
constexpr int S2_LIST = 64;    // per-warp list ring: >= group - 1 + 32
constexpr int S2_SEGS = 64;    // bin segments reaching a tile: <= 5 x 5 x 2 for P <= 16
constexpr int S2_FOLD = 512;   // FP32 partial sums cover this many of a warp's particles

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

template <typename Acc>
struct Spread2Smem {
    Spread2Stage<Acc> stage[S2_WARPS][2];
    int2 list[S2_WARPS][S2_LIST];   // (particle, packed grid index)
    int seg_beg[S2_SEGS];
    int seg_pre[S2_SEGS];
    int wsum[S2_WARPS];
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

// The number of candidates of tile lt of system S (the particles of the bin
// segments that reach it), summed over the warp; every lane gets it.
__device__ __forceinline__ int tile_candidates(const SysDev& S, int lt, const int* __restrict__ boff,
                                               int lane)
{
    const int nt = S.nt[0];
    const int tix = lt / (nt * nt), tiy = (lt / nt) % nt, tiz = lt % nt;
    const BinRanges rx = bins_reaching(tix * 16, 16, S.M, S.P, S.nf[0]);
    const BinRanges ry = bins_reaching(tiy * 16, 16, S.M, S.P, S.nf[1]);
    const BinRanges rz = bins_reaching(tiz * 16, 16, S.M, S.P, S.nf[2]);
    const int nx = range_count(rx), ny = range_count(ry);
    int sum = 0;
    for (int u = lane; u < nx * ny * 2; u += 32) {
        const int zr = u & 1, iy = (u >> 1) % ny, ix = (u >> 1) / ny;
        const int bz0 = zr ? rz.b0 : rz.a0, bz1 = zr ? rz.b1 : rz.a1;
        if (bz0 <= bz1) {
            const int kb = S.bin_base + (range_at(rx, ix) * S.nf[1] + range_at(ry, iy)) * S.nf[2];
            sum += boff[kb + bz1 + 1] - boff[kb + bz0];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    return sum;
}

// Parts per tile (one warp per tile: max(1, ceil(candidates / S2_CAP)) for
// the k_spread2 systems, 1 for the others), then, in the block that finishes
// last, their exclusive scan in place: parts[t] = the first part of tile t,
// parts[ntiles] = the number of parts.  More parts than the launch bound
// (which no input reaches: a bin is a candidate of at most two tiles per
// axis) set bit 2 of err.  The block counter is left at zero for the next
// launch.
constexpr int TP_WARPS = 8;

__global__ void __launch_bounds__(TP_WARPS * 32) k_tile_parts(
    const SysDev* __restrict__ sys, const int* __restrict__ tile_prefix, int nsys, int ntiles,
    const int* __restrict__ boff, int* parts, unsigned* counter, int bound, int* err)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * TP_WARPS + warp;
    if (tile < ntiles) {
        const SysDev& S = sys[find_sys(tile_prefix, nsys, tile)];
        int n = 1;
        if (S.path & PATH_TILE_SPREAD) {
            const int c = tile_candidates(S, tile - S.tile_base, boff, lane);
            n = max(1, (c + S2_CAP - 1) / S2_CAP);
        }
        if (lane == 0) parts[tile] = n;
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
}

template <typename Acc>
__global__ void __launch_bounds__(S2_THREADS, sizeof(Acc) == 4 ? SE_S2_MIN_BLOCKS : 3) k_spread2(
    const SysDev* __restrict__ sys, const int* __restrict__ tile_prefix, int nsys,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const Acc* __restrict__ rows, const int* __restrict__ boff, double* __restrict__ grid,
    const int* __restrict__ tile_parts, int ntiles, int* __restrict__ tile_done,
    double* __restrict__ slab, int slab_slots, int* __restrict__ err)
{
    constexpr bool FOLD = sizeof(Acc) == 4;
    constexpr int G = s2_group<Acc>();
    constexpr int V = 16 / sizeof(Acc);   // entries per 16-byte copy
    __shared__ __align__(16) Spread2Smem<Acc> sm;
    __shared__ int folds;   // this CTA finished its tile's parts last

    // ---- the part this CTA sums: tile = the last t with tile_parts[t] <= item
    const int item = blockIdx.x;
    if (item >= tile_parts[ntiles]) return;
    int tile = 0;
    {
        int hi = ntiles - 1;
        while (tile < hi) {
            const int mid = (tile + hi + 1) >> 1;
            if (tile_parts[mid] <= item) tile = mid;
            else hi = mid - 1;
        }
    }
    const int ipart = item - tile_parts[tile];
    const int nparts = tile_parts[tile + 1] - tile_parts[tile];
    const SysDev& S = sys[find_sys(tile_prefix, nsys, tile)];
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
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wy = warp >> 1, wz = warp & 1;
    const int ly = lane >> 2, lz = (lane & 3) * 2;
    const unsigned ybits = 0xFFu << (8 * wy), zbits = 0xFFu << (8 * wz);

    // ---- the bin segments reaching this tile (at most 5 x 5 x 2) and their prefix
    const BinRanges rx = bins_reaching(x0, 16, M, P, S.nf[0]);
    const BinRanges ry = bins_reaching(y0, 16, M, P, S.nf[1]);
    const BinRanges rz = bins_reaching(z0, 16, M, P, S.nf[2]);
    const int nx = range_count(rx), ny = range_count(ry);
    const int nseg = nx * ny * 2;
    int beg = 0, len = 0;
    if (t < nseg) {
        const int zr = t & 1, iy = (t >> 1) % ny, ix = (t >> 1) / ny;
        const int bz0 = zr ? rz.b0 : rz.a0, bz1 = zr ? rz.b1 : rz.a1;
        if (bz0 <= bz1) {
            const int kb = S.bin_base + (range_at(rx, ix) * S.nf[1] + range_at(ry, iy)) * S.nf[2];
            beg = boff[kb + bz0];
            len = boff[kb + bz1 + 1] - beg;
        }
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) sm.wsum[warp] = incl;
    __syncthreads();
    int before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < S2_WARPS; w++) {
        const int v = sm.wsum[w];
        before += w < warp ? v : 0;
        total += v;
    }
    if (t < S2_SEGS) {
        sm.seg_beg[t] = beg;
        sm.seg_pre[t] = before + incl - len;
    }
    __syncthreads();   // the last CTA barrier: from here on the warps are independent

    const unsigned pmask = (1u << P) - 1u;   // P <= 16
    const unsigned lanes_before = (1u << lane) - 1u;
    int2* list = sm.list[warp];
    double* gs = grid + S.grid_off;
    const long long gplane = (long long)M * M;
    // part 0 sums into the grid, the others into their slab slot
    // (cells [x][y][z] of the tile, 16^3)
    const long long plane = ipart == 0 ? gplane : 256;
    double* cell0 =
        ipart == 0 ? gs + (long long)x0 * gplane + (long long)(y0 + 8 * wy + ly) * M + z0 + 8 * wz + lz
                  : slab + (long long)(slot0 + ipart - 1) * 4096 + (8 * wy + ly) * 16 + 8 * wz + lz;
    // this part's candidates: [cbeg, cend) of the tile's list
    const int cbeg = ipart * S2_CAP, cend = min(total, cbeg + S2_CAP);

    Spread2Accum<Acc> acc;
    acc.zero();
    int cpos = cbeg, head = 0, tail = 0, buf = 0, pending = 0, since_fold = 0;
    int seg = 0;   // the segment holding candidate cpos
    while (seg + 1 < nseg && sm.seg_pre[seg + 1] <= cpos) seg++;
    bool written = false;
    for (;;) {
        // ---- list at least a group (or every remaining candidate), in order
        while (tail - head < G && cpos < cend) {
            const int pos = cpos + lane;
            int part = -1, pk = 0, sl = seg;   // this lane's segment, found forward
            if (pos < cend) {
                while (sl + 1 < nseg && sm.seg_pre[sl + 1] <= pos) sl++;
                part = sm.seg_beg[sl] + (pos - sm.seg_pre[sl]);
                pk = sg[part];
                // the stencil's cells in this tile, as 16-bit masks per axis
                const int gy = g_of(pk, 1), gz = g_of(pk, 2);
                const int hy = tile_half(gy, tiy, nt, P), hz = tile_half(gz, tiz, nt, P);
                const bool meets = tile_half(g_of(pk, 0), tix, nt, P) >= 0 && hy >= 0 &&
                                   hz >= 0 &&
                                   ((((pmask << (gy & 15)) >> (16 * hy)) & 0xFFFFu) & ybits) &&
                                   ((((pmask << (gz & 15)) >> (16 * hz)) & 0xFFFFu) & zbits);
                if (!meets) part = -1;
            }
            const unsigned keep = __ballot_sync(0xffffffffu, part >= 0);
            if (part >= 0)
                list[(tail + __popc(keep & lanes_before)) & (S2_LIST - 1)] = make_int2(part, pk);
            tail += __popc(keep);
            cpos += 32;
            seg = __reduce_max_sync(0xffffffffu, sl);
        }
        __syncwarp();   // list entries visible to the warp
        // ---- stage the next group: lane l < n copies particle head + l
        const int n = min(G, tail - head);
        if (n > 0) {
            Spread2Stage<Acc>& st = sm.stage[warp][buf];
            if (lane < n) {
                const int2 e = list[(head + lane) & (S2_LIST - 1)];
                const int hx = tile_half(g_of(e.y, 0), tix, nt, P);
                const int hy = tile_half(g_of(e.y, 1), tiy, nt, P);
                const int hz = tile_half(g_of(e.y, 2), tiz, nt, P);
                const Acc* r = rows + (long long)e.x * 96;
#pragma unroll
                for (int k = 0; k < 16; k += V) cp_async16(&st.px[lane][k], r + 16 * hx + k);
#pragma unroll
                for (int k = 0; k < 8; k += V) {
                    cp_async16(&st.py[lane][k], r + 32 + 16 * hy + 8 * wy + k);
                    cp_async16(&st.pz[lane][k], r + 64 + 16 * hz + 8 * wz + k);
                }
                cp_async8(&st.q[lane], &srec[e.x].w);
            }
#if SE_S2_FULL_GROUP
            else if (lane < G) {   // a short (the last) group: zero rows up to G (FP64: 16),
                                   // so every group sums G rows
#pragma unroll
                for (int k = 0; k < 16; k++) st.px[lane][k] = Acc(0);
#pragma unroll
                for (int k = 0; k < 8; k++) st.py[lane][k] = st.pz[lane][k] = Acc(0);
                st.q[lane] = 0.0;
            }
#endif
            cp_async_commit();
            head += n;
        }
        __syncwarp();   // the staged entries are read before the list refills over them
        // ---- the previous group, while this one lands
        if (pending > 0) {
            if (n > 0) cp_async_wait<1>();
            else cp_async_wait<0>();
            __syncwarp();
            Spread2Stage<Acc>& st = sm.stage[warp][buf ^ 1];
            // lane i scales its particle's 8 y entries by the charge, once
            if (lane < pending) {
                const Acc qv = (Acc)st.q[lane];
#pragma unroll
                for (int k = 0; k < 8; k++) st.py[lane][k] = st.py[lane][k] * qv;
            }
            __syncwarp();
#if SE_S2_FULL_GROUP
            // every group holds G rows (a short one padded with zeros, which
            // add exact zeros): one unrolled pass with constant offsets
#pragma unroll
            for (int i = 0; i < G; i++) {
#else
#pragma unroll 2
            for (int i = 0; i < pending; i++) {
#endif
                const Acc y = st.py[i][ly];
                acc.add(st.px[i], y * st.pz[i][lz], y * st.pz[i][lz + 1]);
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
        if (t == 0) folds = atomicAdd(&tile_done[tile], 1) == nparts - 1;
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
