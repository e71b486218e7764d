// se_spread.cuh -- the spread (SE_FGG_grid, SE_fgg.c:3866-4028) with the
// periodic fold (SE_FGG_wrap_fcn, SE_fgg.c:327-352) fused, output-stationary.
// Included inside namespace se by se_solve.cu.
//
// One CTA owns a TX x TY x TZ tile of one system's periodic grid and visits
// every particle whose stencil reaches the tile: the particles of at most
// 7 x 7 x 2 contiguous bin segments, gathered into chunks of CHUNK.  For each
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
    Acc px[CHUNK][TX];
    Acc py[CHUNK][TY];
    Acc pz[CHUNK][TZ];
    unsigned ymask[CHUNK];
    unsigned zmask[CHUNK];
    int pidx[CHUNK];
    int seg_beg[SPREAD_THREADS];
    int seg_pre[SPREAD_THREADS];
    int wsum[SPREAD_WARPS];
};

template <typename Acc>
__global__ void __launch_bounds__(SPREAD_THREADS) k_spread(
    const SysDev* __restrict__ sys, const int* __restrict__ tile_prefix, int nsys,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const Acc* __restrict__ fac, int PS, const int* __restrict__ boff, double* __restrict__ grid)
{
    constexpr bool FOLD = sizeof(Acc) == 4;
    static_assert(TX == 16 && TY == 16 && TZ == 16 && CHUNK == 64 && SPREAD_WARPS == 8,
                  "the factor-row builder assumes 16-cell rows and 64-particle chunks");
    __shared__ __align__(16) SpreadSmem<Acc> sm;

    const int tile = blockIdx.x;
    const SysDev& S = sys[find_sys(tile_prefix, nsys, tile)];
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

    Acc acc[TX];
    double accd[FOLD ? TX : 1];
#pragma unroll
    for (int x = 0; x < TX; x++) acc[x] = Acc(0);
#pragma unroll
    for (int x = 0; x < (FOLD ? TX : 1); x++) accd[x] = 0.0;

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
        // factor rows: warps 2a, 2a+1 build axis a, one lane per particle
        if (warp < 6) {
            const int a = warp >> 1, p = t & 63;
            if (p < n) {
                const int part = sm.pidx[p];
                const int g = g_of(sg[part], a);
                const int o = a == 0 ? x0 : (a == 1 ? y0 : z0);
                const Acc* f = fac + ((long long)part * 3 + a) * PS;
                const Acc scale = a == 0 ? (Acc)srec[part].w : Acc(1);
                Acc* dst = a == 0 ? sm.px[p] : (a == 1 ? sm.py[p] : sm.pz[p]);
                unsigned mask = 0;
                int i = wrap1(o - g, S.M);
#pragma unroll
                for (int xo = 0; xo < 16; xo++) {
                    Acc v = Acc(0);
                    if (o + xo < S.M)
                        for (int k = i; k < S.P; k += S.M) v += f[k];
                    dst[xo] = v * scale;
                    mask |= (v != Acc(0)) ? (1u << xo) : 0u;
                    if (++i >= S.M) i -= S.M;
                }
                if (a == 1) sm.ymask[p] = mask;
                if (a == 2) sm.zmask[p] = mask;
            }
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
                const Acc c = sm.py[p][ly] * sm.pz[p][lz];
                const Acc* px = sm.px[p];
#pragma unroll
                for (int x = 0; x < TX; x++) acc[x] = fma(px[x], c, acc[x]);
            }
        }
        if (FOLD) {
#pragma unroll
            for (int x = 0; x < TX; x++) {
                accd[x] += (double)acc[x];
                acc[x] = Acc(0);
            }
        }
    }

    // ---- write the tile (every cell once; cells past M belong to no tile)
    const int gy = y0 + ly, gz = z0 + lz;
    if (gy >= S.M || gz >= S.M) return;
    double* gs = grid + S.grid_off;
#pragma unroll
    for (int x = 0; x < TX; x++) {
        const int gx = x0 + x;
        if (gx < S.M)
            gs[((long long)gx * S.M + gy) * S.M + gz] = FOLD ? accd[x] : (double)acc[x];
    }
}
