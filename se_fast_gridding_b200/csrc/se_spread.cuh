// se_spread.cuh -- the spread (SE_FGG_grid, SE_fgg.c:3866-4028) with the
// periodic fold (SE_FGG_wrap_fcn, SE_fgg.c:327-352) fused, output-stationary.
// Included inside namespace se by se_solve.cu.
//
// One CTA owns a TX x TY x TZ tile of one system's periodic grid and visits
// every particle whose stencil reaches the tile: the particles of at most
// 7 x 7 x 2 contiguous bin segments, gathered into chunks of spread_chunk<Acc>().  For each
// chunk the CTA builds the factor rows of its particles restricted to the
// tile (px[TX], py[TY], pz[TZ], zero outside the stencil, the charge folded
// into px) from the precomputed factors, with bit masks of the nonzero y and
// z entries.  Each warp owns a WY x WZ block of (y, z) cells (one per lane)
// and TX x-cells per lane in registers; it skips, as a whole warp, every
// particle whose stencil misses its block, and otherwise adds
// px[x] * (py[y] pz[z]) to its TX accumulators.  Every cell is written once
// at the end: no atomics, a deterministic order of summation, and the fold is
// the index arithmetic of the factor rows.
//
// FP32 (compensated): after every chunk the FP32 partial sums of a cell are
// added into an FP64 register accumulator.

// Up to two fine-bin ranges whose corners reach the output cells [o, o+T).
struct BinRanges {
    int a0, a1, b0, b1;   // [a0,a1] and [b0,b1]; b0 > b1 when absent
};

__device__ __forceinline__ BinRanges bins_reaching(int o, int T, int M, int P, int nf)
{
    BinRanges r;
    const int Ta = min(T, M - o);
    const int len = Ta + P - 1;   // corners g with (g + i) mod M in the tile, i < P
    if (len >= M) {
        r.a0 = 0; r.a1 = nf - 1; r.b0 = 1; r.b1 = 0;
        return r;
    }
    const int start = pmod(o - P + 1, M);
    const int end = start + len - 1;
    if (end < M) {
        r.a0 = start / FB; r.a1 = end / FB; r.b0 = 1; r.b1 = 0;
    } else {
        const int e2 = end - M;
        r.a0 = start / FB; r.a1 = nf - 1;
        r.b0 = 0; r.b1 = e2 / FB;
        if (r.b1 >= r.a0) { r.a0 = 0; r.a1 = nf - 1; r.b0 = 1; r.b1 = 0; }
    }
    return r;
}

__device__ __forceinline__ int range_count(const BinRanges& r)
{
    return (r.a1 - r.a0 + 1) + (r.b1 >= r.b0 ? r.b1 - r.b0 + 1 : 0);
}

__device__ __forceinline__ int range_at(const BinRanges& r, int k)
{
    const int na = r.a1 - r.a0 + 1;
    return k < na ? r.a0 + k : r.b0 + (k - na);
}

template <typename Acc>
struct SpreadSmem {
    Acc px[spread_chunk<Acc>()][TX];
    Acc py[spread_chunk<Acc>()][TY];
    Acc pz[spread_chunk<Acc>()][TZ];
    unsigned ymask[spread_chunk<Acc>()];
    unsigned zmask[spread_chunk<Acc>()];
    int pidx[spread_chunk<Acc>()];
    int seg_beg[SPREAD_THREADS];
    int seg_pre[SPREAD_THREADS];
    int wsum[SPREAD_WARPS];
    // FP64 fold of the FP32 chunk sums, [cell x][thread] (FP32 path only)
    double fold[sizeof(Acc) == 4 ? TX : 1][SPREAD_THREADS];
};

// The TX accumulators of one lane.
template <typename Acc>
struct SpreadAccum;

template <>
struct SpreadAccum<float> {
    float2 v[TX / 2];   // packed pairs (x = 2m, 2m + 1)
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int m = 0; m < TX / 2; m++) v[m] = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void add(const float* px, float c)
    {
        const float2 cc = f32x2(c, c);
        const float4* p4 = reinterpret_cast<const float4*>(px);
#pragma unroll
        for (int m = 0; m < TX / 4; m++) {
            float2 lo, hi;
            f32x2_split(p4[m], lo, hi);
            v[2 * m] = ffma2(lo, cc, v[2 * m]);
            v[2 * m + 1] = ffma2(hi, cc, v[2 * m + 1]);
        }
    }
    __device__ __forceinline__ void fold(SpreadSmem<float>& sm, int t)
    {
#pragma unroll
        for (int m = 0; m < TX / 2; m++) {
            sm.fold[2 * m][t] += (double)v[m].x;
            sm.fold[2 * m + 1][t] += (double)v[m].y;
            v[m] = make_float2(0.f, 0.f);
        }
    }
    __device__ __forceinline__ double result(const SpreadSmem<float>& sm, int t, int x) const
    {
        return sm.fold[x][t];
    }
};

template <>
struct SpreadAccum<double> {
    double v[TX];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int x = 0; x < TX; x++) v[x] = 0.0;
    }
    __device__ __forceinline__ void add(const double* px, double c)
    {
#pragma unroll
        for (int x = 0; x < TX; x++) v[x] = fma(px[x], c, v[x]);
    }
    __device__ __forceinline__ void fold(SpreadSmem<double>&, int) {}
    __device__ __forceinline__ double result(const SpreadSmem<double>&, int, int x) const
    {
        return v[x];
    }
};

template <typename Acc>
__global__ void __launch_bounds__(SPREAD_THREADS, sizeof(Acc) == 4 ? 4 : 2) k_spread(
    const SysDev* __restrict__ sys, const int* __restrict__ tile_prefix, int nsys,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const Acc* __restrict__ fac, int PS, const int* __restrict__ boff, double* __restrict__ grid)
{
    constexpr bool FOLD = sizeof(Acc) == 4;
    static_assert(TX == 16 && TY == 16 && TZ == 16 && SPREAD_WARPS == 8,
                  "the factor-row builder assumes 16-cell rows");
    constexpr int CHUNK = spread_chunk<Acc>();
    __shared__ __align__(16) SpreadSmem<Acc> sm;

    const int tile = blockIdx.x;
    const SysDev& S = sys[find_sys(tile_prefix, nsys, tile)];
    if (S.path & PATH_TILE_SPREAD) return;   // k_spread2 covers this system
    const int lt = tile - S.tile_base;
    const int x0 = (lt / (S.nt[1] * S.nt[2])) * TX;
    const int y0 = ((lt / S.nt[2]) % S.nt[1]) * TY;
    const int z0 = (lt % S.nt[2]) * TZ;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // this warp's (y, z) lane block and this lane's cell in it
    const int wyb = (warp / (TZ / WZ)) * WY, wzb = (warp % (TZ / WZ)) * WZ;
    const int ly = wyb + lane / WZ, lz = wzb + lane % WZ;
    const unsigned ybits = ((1u << WY) - 1u) << wyb, zbits = ((1u << WZ) - 1u) << wzb;

    // ---- the bin segments reaching this tile, one per thread, and their prefix
    const BinRanges rx = bins_reaching(x0, TX, S.M, S.P, S.nf[0]);
    const BinRanges ry = bins_reaching(y0, TY, S.M, S.P, S.nf[1]);
    const BinRanges rz = bins_reaching(z0, TZ, S.M, S.P, S.nf[2]);
    const int nx = range_count(rx), ny = range_count(ry);
    int beg = 0, len = 0;
    if (t < nx * ny * 2) {
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
    for (int w = 0; w < SPREAD_WARPS; w++) {
        const int v = sm.wsum[w];
        before += w < warp ? v : 0;
        total += v;
    }
    sm.seg_beg[t] = beg;
    sm.seg_pre[t] = before + incl - len;

    // accumulators: FP32 as 8 packed pairs (fma.rn.f32x2) with the FP64 fold
    // of the chunk sums in shared memory; FP64 in registers
    SpreadAccum<Acc> acc;
    acc.zero();
    if (FOLD)
        for (int x = 0; x < TX; x++) sm.fold[x][t] = 0.0;

    for (int c0 = 0; c0 < total; c0 += CHUNK) {
        const int n = min(CHUNK, total - c0);
        __syncthreads();   // segment table ready / previous chunk consumed
        if (t < n) {       // chunk slot -> particle: last segment starting at or before pos
            const int pos = c0 + t;
            int lo = 0, hi = SPREAD_THREADS - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sm.seg_pre[mid] <= pos) lo = mid;
                else hi = mid - 1;
            }
            sm.pidx[t] = sm.seg_beg[lo] + (pos - sm.seg_pre[lo]);
        }
        __syncthreads();
        // factor rows: lane = (particle, quad of 4 cells); a warp instruction
        // stores 8 particles' rows of one axis as float4-wide quads, the
        // minimum number of shared-memory wavefronts for the bytes written
        for (int u = t; u < 3 * 4 * CHUNK; u += SPREAD_THREADS) {
            const int a = (u >> 2) / CHUNK, p = (u >> 2) - a * CHUNK, x4 = 4 * (u & 3);
            Acc v[4] = {Acc(0), Acc(0), Acc(0), Acc(0)};
            unsigned nib = 0;
            if (p < n) {
                const int part = sm.pidx[p];
                const int g = g_of(sg[part], a);
                const int o = a == 0 ? x0 : (a == 1 ? y0 : z0);
                const Acc* f = fac + ((long long)part * 3 + a) * PS;
                int k0 = wrap1(o + x4 - g, S.M);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    if (o + x4 + e < S.M)
                        for (int k = k0; k < S.P; k += S.M) v[e] += f[k];
                    if (++k0 >= S.M) k0 -= S.M;
                }
                if (a == 0) {
                    const Acc qw = (Acc)srec[part].w;
#pragma unroll
                    for (int e = 0; e < 4; e++) v[e] *= qw;
                }
#pragma unroll
                for (int e = 0; e < 4; e++) nib |= (v[e] != Acc(0)) ? (1u << e) : 0u;
                Acc* row = (a == 0 ? sm.px[p] : (a == 1 ? sm.py[p] : sm.pz[p])) + x4;
                if constexpr (sizeof(Acc) == 4) {
                    *reinterpret_cast<float4*>(row) = make_float4(v[0], v[1], v[2], v[3]);
                } else {
                    reinterpret_cast<double2*>(row)[0] = make_double2(v[0], v[1]);
                    reinterpret_cast<double2*>(row)[1] = make_double2(v[2], v[3]);
                }
            }
            // 16-bit row mask of the particle from the four lanes of its quads
            unsigned m = nib << x4;
            m |= __shfl_xor_sync(0xffffffffu, m, 1);
            m |= __shfl_xor_sync(0xffffffffu, m, 2);
            if (a > 0 && x4 == 0 && p < n) (a == 1 ? sm.ymask : sm.zmask)[p] = m;
        }
        __syncthreads();
        // this warp's particles: the stencil meets its (y, z) lane block
        for (int base = 0; base < n; base += 32) {
            const int q = base + lane;
            const bool act = q < n && (sm.ymask[q] & ybits) && (sm.zmask[q] & zbits);
            unsigned bits = __ballot_sync(0xffffffffu, act);
            while (bits) {
                const int p = base + __ffs(bits) - 1;
                bits &= bits - 1;
                acc.add(sm.px[p], sm.py[p][ly] * sm.pz[p][lz]);
            }
        }
        if (FOLD) acc.fold(sm, t);
    }

    // ---- write the tile (every cell once; cells past M belong to no tile)
    if (FOLD) __syncwarp();
    const int gy = y0 + ly, gz = z0 + lz;
    if (gy >= S.M || gz >= S.M) return;
    double* gs = grid + S.grid_off;
#pragma unroll
    for (int x = 0; x < TX; x++) {
        const int gx = x0 + x;
        if (gx < S.M) gs[((long long)gx * S.M + gy) * S.M + gz] = acc.result(sm, t, x);
    }
}
