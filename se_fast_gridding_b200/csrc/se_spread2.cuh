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
// One CTA of 4 warps owns one 16^3 tile.  It streams the particles of the
// bin segments that reach the tile, keeps only those whose stencil really
// meets it (in candidate order, through a ring queue: deterministic), and
// takes them 64 at a time: their tile rows go to shared memory (the charge
// folded into the x row), each warp lists the particles whose y rows meet its
// 4 y planes, and each lane adds px[x] * (py[y] pz[z]) into 16 x 2 cells (all
// 16 x of its (y, z) and (y, z + 1)).  Every cell is written once: no atomics
// and a fixed order of summation.  FP32: fma.rn.f32x2 on the packed cells,
// and after every 128 particles (two chunks) the FP32 sums are added into
// FP64 in shared memory.

constexpr int S2_WARPS = 4;
constexpr int S2_THREADS = S2_WARPS * 32;
constexpr int S2_CHUNK = 64;
constexpr int S2_RING = 256;   // > S2_CHUNK + S2_THREADS
constexpr int S2_SEGS = 64;    // bin segments reaching a tile: <= 5 x 5 x 2 for P <= 16

template <typename Acc>
struct Spread2Smem {
    Acc px[S2_CHUNK][16];
    Acc py[S2_CHUNK][16];
    Acc pz[S2_CHUNK][16];
    unsigned ymask[S2_CHUNK];
    int list[S2_WARPS][S2_CHUNK];
    int ring[S2_RING];
    int seg_beg[S2_SEGS];
    int seg_pre[S2_SEGS];
    int wsum[S2_WARPS];
    double fold[sizeof(Acc) == 4 ? 32 : 1][S2_THREADS];
};

// The 32 cells of one lane: 16 x for z and for z + 1.
template <typename Acc>
struct Spread2Accum;

template <>
struct Spread2Accum<float> {
    unsigned long long a[8], b[8];   // packed x pairs for z and z + 1
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int m = 0; m < 8; m++) a[m] = b[m] = 0ull;
    }
    __device__ __forceinline__ void add(const float* px, float c0, float c1)
    {
        const unsigned long long k0 = f32x2(c0, c0), k1 = f32x2(c1, c1);
        const ulonglong2* p2 = reinterpret_cast<const ulonglong2*>(px);
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const ulonglong2 w = p2[m];
            a[2 * m] = ffma2(w.x, k0, a[2 * m]);
            a[2 * m + 1] = ffma2(w.y, k0, a[2 * m + 1]);
            b[2 * m] = ffma2(w.x, k1, b[2 * m]);
            b[2 * m + 1] = ffma2(w.y, k1, b[2 * m + 1]);
        }
    }
    // cell c: x = c >> 1, z + (c & 1)
    __device__ __forceinline__ void fold(Spread2Smem<float>& sm, int t)
    {
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const float2 u = f32x2_unpack(a[m]), v = f32x2_unpack(b[m]);
            sm.fold[4 * m + 0][t] += (double)u.x;
            sm.fold[4 * m + 1][t] += (double)v.x;
            sm.fold[4 * m + 2][t] += (double)u.y;
            sm.fold[4 * m + 3][t] += (double)v.y;
            a[m] = b[m] = 0ull;
        }
    }
    __device__ __forceinline__ double2 result(const Spread2Smem<float>& sm, int t, int x) const
    {
        return make_double2(sm.fold[2 * x][t], sm.fold[2 * x + 1][t]);
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
    __device__ __forceinline__ void fold(Spread2Smem<double>&, int) {}
    __device__ __forceinline__ double2 result(const Spread2Smem<double>&, int, int x) const
    {
        return make_double2(a[x], b[x]);
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

template <typename Acc>
__global__ void __launch_bounds__(S2_THREADS, sizeof(Acc) == 4 ? 4 : 3) k_spread2(
    const SysDev* __restrict__ sys, const int* __restrict__ tile_prefix, int nsys,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const Acc* __restrict__ rows, const int* __restrict__ boff, double* __restrict__ grid)
{
    constexpr bool FOLD = sizeof(Acc) == 4;
    __shared__ __align__(16) Spread2Smem<Acc> sm;

    const int tile = blockIdx.x;
    const SysDev& S = sys[find_sys(tile_prefix, nsys, tile)];
    if (!(S.path & PATH_TILE_SPREAD)) return;   // k_spread covers this system
    const int nt = S.nt[0], P = S.P, M = S.M;
    const int lt = tile - S.tile_base;
    const int tix = lt / (nt * nt), tiy = (lt / nt) % nt, tiz = lt % nt;
    const int x0 = tix * 16, y0 = tiy * 16, z0 = tiz * 16;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int ly = warp * 4 + (lane >> 3), lz = (lane & 7) * 2;
    const unsigned wbits = 0xFu << (warp * 4);

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

    Spread2Accum<Acc> acc;
    acc.zero();
    if (FOLD)
        for (int c = 0; c < 32; c++) sm.fold[c][t] = 0.0;
    const unsigned pmask = (P >= 32) ? 0xffffffffu : ((1u << P) - 1u);

    int head = 0, tail = 0, nfold = 0;
    for (int cb = 0; cb < total; cb += S2_THREADS) {
        __syncthreads();   // segment table ready; wsum free
        // ---- candidates: keep the particles whose stencil meets the tile
        const int pos = cb + t;
        int part = -1;
        if (pos < total) {
            int lo = 0, hi = nseg - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sm.seg_pre[mid] <= pos) lo = mid;
                else hi = mid - 1;
            }
            part = sm.seg_beg[lo] + (pos - sm.seg_pre[lo]);
            const int pk = sg[part];
            if (tile_half(g_of(pk, 0), tix, nt, P) < 0 || tile_half(g_of(pk, 1), tiy, nt, P) < 0 ||
                tile_half(g_of(pk, 2), tiz, nt, P) < 0)
                part = -1;
        }
        const unsigned keep = __ballot_sync(0xffffffffu, part >= 0);
        if (lane == 0) sm.wsum[warp] = __popc(keep);
        __syncthreads();
        int wbefore = 0, added = 0;
#pragma unroll
        for (int w = 0; w < S2_WARPS; w++) {
            const int v = sm.wsum[w];
            wbefore += w < warp ? v : 0;
            added += v;
        }
        if (part >= 0)
            sm.ring[(tail + wbefore + __popc(keep & ((1u << lane) - 1u))) & (S2_RING - 1)] = part;
        tail += added;
        const bool last = cb + S2_THREADS >= total;

        // ---- full chunks (and the remainder after the last candidates)
        while (tail - head >= S2_CHUNK || (last && tail > head)) {
            const int n = min(S2_CHUNK, tail - head);
            __syncthreads();   // ring written; previous chunk's rows consumed
            for (int it = t; it < 3 * n; it += S2_THREADS) {
                const int a = it / n, p = it - a * n;
                const int part = sm.ring[(head + p) & (S2_RING - 1)];
                const int ga = g_of(sg[part], a);
                const int h = tile_half(ga, a == 0 ? tix : (a == 1 ? tiy : tiz), nt, P);
                if (a == 1) sm.ymask[p] = ((pmask << (ga & 15)) >> (16 * h)) & 0xFFFFu;
                const Acc* src = rows + ((long long)part * 3 + a) * 32 + 16 * h;
                Acc* dst = a == 0 ? sm.px[p] : (a == 1 ? sm.py[p] : sm.pz[p]);
                if constexpr (sizeof(Acc) == 4) {
                    const float4* s4 = reinterpret_cast<const float4*>(src);
                    float4* d4 = reinterpret_cast<float4*>(dst);
                    const float qw = a == 0 ? (float)srec[part].w : 1.0f;
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        float4 v = __ldg(s4 + k);
                        v.x *= qw; v.y *= qw; v.z *= qw; v.w *= qw;
                        d4[k] = v;
                    }
                } else {
                    const double2* s2 = reinterpret_cast<const double2*>(src);
                    double2* d2 = reinterpret_cast<double2*>(dst);
                    const double qw = a == 0 ? srec[part].w : 1.0;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        double2 v = __ldg(s2 + k);
                        v.x *= qw; v.y *= qw;
                        d2[k] = v;
                    }
                }
            }
            __syncthreads();
            // this warp's particles: y rows meeting its 4 y planes
            int cnt = 0;
            for (int base = 0; base < n; base += 32) {
                const int q = base + lane;
                const bool act = q < n && (sm.ymask[q] & wbits);
                const unsigned bits = __ballot_sync(0xffffffffu, act);
                if (act) sm.list[warp][cnt + __popc(bits & ((1u << lane) - 1u))] = q;
                cnt += __popc(bits);
            }
            __syncwarp();
            for (int i = 0; i < cnt; i++) {
                const int p = sm.list[warp][i];
                const Acc y = sm.py[p][ly];
                const Acc c0 = y * sm.pz[p][lz], c1 = y * sm.pz[p][lz + 1];
                acc.add(sm.px[p], c0, c1);
            }
            if (FOLD && (++nfold & 1) == 0) acc.fold(sm, t);
            head += n;
        }
    }

    if (FOLD) acc.fold(sm, t);
    // ---- write the tile: 16 x of (y, z) and (y, z + 1) per lane
    double* gs = grid + S.grid_off;
    const long long row = ((long long)(y0 + ly)) * M + z0 + lz;
#pragma unroll
    for (int x = 0; x < 16; x++)
        *reinterpret_cast<double2*>(gs + (long long)(x0 + x) * M * M + row) = acc.result(sm, t, x);
}
