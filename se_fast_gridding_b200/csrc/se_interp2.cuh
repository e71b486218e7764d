// se_interp2.cuh -- interpolation (SE_FGG_int / SE_FGG_int_force,
// SE_fgg.c:968-1100) with the periodic unfold (SE_FGG_extend_fcn,
// SE_fgg.c:417-443) fused, for the systems k_spread2 serves (whole 16^3
// tiles, P <= 16).  Included inside namespace se by se_solve.cu after
// se_interp.cuh.
//
// One CTA per fine bin (8^3 stencil corners), or per pair of z-adjacent
// bins where bins are sparse and the larger window still leaves three CTAs
// per SM (FP32).  The
// window, E = 7 + P cells per axis in x and y and EZ = 8 zb + P rounded up
// to 4 in z (zb = 1 or 2 bins), is copied
// from the grid (a FP32 copy of it on the FP32 path) by cp.async, a 4-cell
// group at a time: the window starts on a multiple of 8 in every axis and M
// is a multiple of 16, so every group is contiguous even where the window
// wraps.  One warp per particle; lane l takes the (x, y) columns l, l + 32,
// ... (FP32 with P not dividing 32: a whole x row, interp2_rows_f32) and
// sums each column over z in pairs: one 8-byte (FP32) or 16-byte (FP64)
// shared load of two neighbouring cells feeds two packed FMAs per
// accumulator against the particle's z weights, which are zero-padded pairs
// in registers aligned to the window.  Columns combine with the x (and y)
// weights in the working precision; the lanes' sums are reduced in FP64 with
// shuffles (the four FORCE sums of the FP32 kernel together, warp_sum4).
// FP32 warps on x rows copy the next particle's record and factor rows into
// shared memory by cp.async while they sum the current one; warps on columns
// load a particle's three factor rows whole, entry l in lane l, beside its
// record, and take the factors from the loading lanes by shuffles.
//
// Shared-memory pitches (row Ep, plane PL) come from the host, chosen so that
// the pair loads of one instruction fall in distinct banks.

constexpr int I2_WARPS = 8;
#ifndef SE_I2_ZMERGE
#define SE_I2_ZMERGE 1   // windows of two z-adjacent bins where they fit
#endif

template <typename T>
struct Interp2Warp {
    T wx[16], fx[16], wy[16], fy[16];   // x, y weights and force weights (-c u)
    __align__(16) T wz[32];             // z weights shifted to window index
    __align__(16) T fz[32];
};

// Two neighbouring window cells and the matching weights.
template <typename T>
struct Pair;

template <>
struct Pair<float> {
    using V = float2;
    __device__ __forceinline__ static V load(const float* p)
    {
        return *reinterpret_cast<const V*>(p);
    }
    __device__ __forceinline__ static V fma(V a, V b, V c) { return ffma2(a, b, c); }
    __device__ __forceinline__ static float sum(V v) { return v.x + v.y; }
    __device__ __forceinline__ static V zero() { return make_float2(0.f, 0.f); }
};

template <>
struct Pair<double> {
    using V = double2;
    __device__ __forceinline__ static V load(const double* p)
    {
        return *reinterpret_cast<const double2*>(p);
    }
    __device__ __forceinline__ static V fma(V a, V b, V c)
    {
        return make_double2(::fma(a.x, b.x, c.x), ::fma(a.y, b.y, c.y));
    }
    __device__ __forceinline__ static double sum(V v) { return v.x + v.y; }
    __device__ __forceinline__ static V zero() { return make_double2(0.0, 0.0); }
};

// The warp's sums of four values, in lane 0: the first two levels halve the
// vector (each lane keeps two of the four, then one, and adds its partner's
// copy of those), the last three add the one kept, and lanes 8, 16, 24 hand
// lane 0 the sums of the other three.
__device__ __forceinline__ void warp_sum4(double& v0, double& v1, double& v2, double& v3)
{
    const int lane = threadIdx.x & 31;
    const bool h16 = lane & 16, h8 = lane & 8;
    const double k0 = h16 ? v2 : v0, k1 = h16 ? v3 : v1;
    const double w0 = k0 + __shfl_xor_sync(0xffffffffu, h16 ? v0 : v2, 16);
    const double w1 = k1 + __shfl_xor_sync(0xffffffffu, h16 ? v1 : v3, 16);
    double u = (h8 ? w1 : w0) + __shfl_xor_sync(0xffffffffu, h8 ? w0 : w1, 8);
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
    // lane l now holds the sum of value 2 (l >> 4 & 1) + (l >> 3 & 1)
    v0 = u;
    v1 = __shfl_sync(0xffffffffu, u, 8);
    v2 = __shfl_sync(0xffffffffu, u, 16);
    v3 = __shfl_sync(0xffffffffu, u, 24);
}

// z extent of the staged window of zb z-adjacent bins: the pairs of any
// stencil start r2 < 8 zb fit.
__host__ __device__ constexpr int interp2_ez(int P, int zb = 1) { return (FB * zb + P + 3) & ~3; }

// FP32 rows of x (interp2_rows_f32): the next particle's record, packed
// corner, input index and factor rows, copied by cp.async into a per-warp
// slot while the warp sums the current particle (two slots, alternating), so
// the global-load latency of each particle's data is not waited for.  (The
// column mapping of P = 8 and 16 measured 8% and 1.5% slower with it, P = 12
// 3% faster.)
#ifndef SE_I2_PREFETCH
#define SE_I2_PREFETCH 1
#endif
#ifndef SE_I2_ASYNC_STAGE
#define SE_I2_ASYNC_STAGE 1
#endif

struct __align__(16) Interp2Next {
    float rows[2][96];
    double4 rec[2];
    int pk[2], orig[2];
};

__device__ __forceinline__ Interp2Next* interp2_next_slots()
{
    __shared__ Interp2Next slots[I2_WARPS];
    return slots;
}

__device__ __forceinline__ void cp_async4(void* sdst, const void* gsrc)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}

// Lanes 0-23 copy the 384-byte factor rows of particle p, 24-25 its record,
// 26 its corner, 27 its input index into slot `slot`.
__device__ __forceinline__ void interp2_fetch(Interp2Next& nx, int slot, int p,
                                              const double4* __restrict__ srec,
                                              const int* __restrict__ sg,
                                              const int* __restrict__ sperm,
                                              const float* __restrict__ rows, int lane)
{
    if (lane < 24)
        cp_async16(&nx.rows[slot][4 * lane], rows + (long long)p * 96 + 4 * lane);
    else if (lane < 26)
        cp_async16(reinterpret_cast<char*>(&nx.rec[slot]) + 16 * (lane - 24),
                   reinterpret_cast<const char*>(srec + p) + 16 * (lane - 24));
    else if (lane == 26)
        cp_async4(&nx.pk[slot], sg + p);
    else if (lane == 27)
        cp_async4(&nx.orig[slot], sperm + p);
}

// The FP32 particle loop for P that does not divide 32 (P = 12 among the
// configurations; P = 8 and 16 take the column mapping of k_interp2, which
// measured 17% and 2% faster there): lane l < k P (k = 32 / P groups of P lanes) takes
// the x row i = l % P of the stencil and, in its group g = l / P, the J =
// ceil(P / k) y columns j = g J + jj; the lanes past k P repeat group k - 1
// with zero weights.  A lane's column sums over z (pair loads, packed FMAs
// against the z weights) combine with its own y weights, held in registers,
// and its x weight multiplies the lane's sums once, in FP64, before the warp
// reduction.  Columns past the stencil (j >= P, when k J > P) read the lane's
// last column with zero weights, so every load stays inside the window and
// the runtime-P kernel sums in the same order as the P-specialised ones.
constexpr int I2_JMAX = 8;   // y columns per lane for P <= 16 (k >= 2)

template <int PT, bool FORCE>
__device__ __forceinline__ void interp2_rows_f32(
    const SysDev& S, Interp2Warp<float>& W, const float* tile, int P, int o0, int o1, int o2,
    int pfirst, int pend, const double4* __restrict__ srec, const int* __restrict__ sg,
    const int* __restrict__ sperm, const float* __restrict__ rows, double* __restrict__ out,
    double* __restrict__ phi_out, int Ep, int PL)
{
    using PV = Pair<float>;
    using VT = float2;
    const int lane = threadIdx.x & 31;
    constexpr int NQ = PT ? PT / 2 + 1 : 9;
    const int nq = P / 2 + 1;
    constexpr int KC = PT ? 32 / PT : 1;
    constexpr int JC = PT ? (PT + KC - 1) / KC : I2_JMAX;
    const int k = PT ? KC : 32 / P;
    const int J = PT ? JC : (P + k - 1) / k;
    const int i = lane % P;
    const int g = min(lane / P, k - 1);
    const bool active = lane < k * P;
    // the lane's last column inside the stencil
    const int jlast = min(J, P - g * J) - 1;
    Interp2Next& nx = interp2_next_slots()[threadIdx.x >> 5];
    if (SE_I2_PREFETCH) {
        if (pfirst < pend) interp2_fetch(nx, 0, pfirst, srec, sg, sperm, rows, lane);
        cp_async_commit();
    }
    int slot = 0;
    for (int p = pfirst; p < pend; p += I2_WARPS, slot ^= 1) {
        double4 rc;
        int pk, orig;
        const float* rb;
        if (SE_I2_PREFETCH) {
            if (p + I2_WARPS < pend)
                interp2_fetch(nx, slot ^ 1, p + I2_WARPS, srec, sg, sperm, rows, lane);
            cp_async_commit();
            cp_async_wait<1>();
            __syncwarp();
            rc = nx.rec[slot];
            pk = nx.pk[slot];
            orig = nx.orig[slot];
            rb = nx.rows[slot];
        } else {
            rc = srec[p];
            pk = sg[p];
            orig = sperm[p];
            rb = rows + (long long)p * 96;
        }
        const int gx = g_of(pk, 0), gy = g_of(pk, 1), gz = g_of(pk, 2);
        const int r0 = gx - o0, r1 = gy - o1, r2 = gz - o2;
        W.wz[lane] = 0.f;
        W.fz[lane] = 0.f;
        __syncwarp();
        if (lane < P) {
            const double off = (S.lo + lane) * S.h;
            const float vx = rb[(gx & 15) + lane], vy = rb[32 + (gy & 15) + lane],
                        vz = rb[64 + (gz & 15) + lane];
            W.wx[lane] = vx;
            W.wy[lane] = vy;
            W.wz[r2 + lane] = vz;
            if (FORCE) {
                W.fx[lane] = (float)((double)vx * (-S.c * (rc.x - off)));
                W.fy[lane] = (float)((double)vy * (-S.c * (rc.y - off)));
                W.fz[r2 + lane] = (float)((double)vz * (-S.c * (rc.z - off)));
            }
        }
        __syncwarp();
        const int q0 = r2 >> 1;
        VT wz2[NQ], fz2[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            if (PT || q < nq) {
                wz2[q] = PV::load(W.wz + 2 * (q0 + q));
                fz2[q] = FORCE ? PV::load(W.fz + 2 * (q0 + q)) : PV::zero();
            }
        }
        const float wxi = active ? W.wx[i] : 0.f;
        const float fxi = (FORCE && active) ? W.fx[i] : 0.f;
        float wy[JC], fy[JC];
#pragma unroll
        for (int jj = 0; jj < JC; jj++) {
            const bool ok = jj < J && jj <= jlast;
            wy[jj] = ok ? W.wy[g * J + jj] : 0.f;
            fy[jj] = (FORCE && ok) ? W.fy[g * J + jj] : 0.f;
        }
        const float* col = tile + (r0 + i) * PL + (r1 + g * J) * Ep + 2 * q0;
        float a_pot = 0.f, a_fy = 0.f, a_fz = 0.f;
        auto columns = [&](auto nqc) {
            constexpr int NQC = decltype(nqc)::value;
#pragma unroll
            for (int jj = 0; jj < JC; jj++) {
                if (!PT && jj >= J) break;
                const float* cj = col + (PT && KC * JC == PT ? jj : min(jj, jlast)) * Ep;
                VT s0 = PV::zero(), s1 = PV::zero();
#pragma unroll
                for (int q = 0; q < NQC; q++) {
                    if (PT || q < nq) {
                        const VT g2 = PV::load(cj + 2 * q);
                        s0 = PV::fma(g2, wz2[q], s0);
                        if (FORCE) s1 = PV::fma(g2, fz2[q], s1);
                    }
                }
                const float t0 = PV::sum(s0);
                a_pot = fmaf(t0, wy[jj], a_pot);
                if (FORCE) {
                    a_fy = fmaf(t0, fy[jj], a_fy);
                    a_fz = fmaf(PV::sum(s1), wy[jj], a_fz);
                }
            }
        };
        // an even stencil that starts on a pair spans P/2 pairs, not P/2 + 1
        // (a warp-uniform choice: the pair the other form adds is zero)
        if (PT != 0 && PT % 2 == 0 && (r2 & 1) == 0)
            columns(std::integral_constant<int, (PT ? PT / 2 : 1)>{});
        else
            columns(std::integral_constant<int, NQ>{});
        double d_pot = (double)a_pot * (double)wxi;
        double d_fx = 0, d_fy = 0, d_fz = 0;
        if (FORCE) {
            d_fx = (double)a_pot * (double)fxi;
            d_fy = (double)a_fy * (double)wxi;
            d_fz = (double)a_fz * (double)wxi;
            warp_sum4(d_pot, d_fx, d_fy, d_fz);
        } else {
            d_pot = warp_sum(d_pot);
        }
        if (lane == 0)
            interp_store(S, orig - S.part_off, rc.w, d_pot, d_fx, d_fy, d_fz,
                         S.mode == SE_FORCE, out, phi_out);
        __syncwarp();   // the slot is read before it is refilled
    }
    if (SE_I2_PREFETCH) cp_async_wait<0>();
}

template <typename T, int PT, bool FORCE>
__device__ __forceinline__ void interp2_columns(
    const SysDev& S, Interp2Warp<T>& W, const T* tile, int P, int o0, int o1, int o2,
    int pfirst, int pend, const double4* __restrict__ srec, const int* __restrict__ sg,
    const int* __restrict__ sperm, const T* __restrict__ rows, double* __restrict__ out,
    double* __restrict__ phi_out, int Ep, int PL, bool JFIX);

// FORCE: the force weights and sums are computed (every system of a batch
// with a FORCE system runs this variant; each stores what its mode asks).
// A launch serves the systems of one stencil (a batch of several stencils
// runs one launch per stencil, each with its window), one CTA per unit of zb
// z-adjacent bins: tab[u] is unit u's system and tab[units + u] its first
// bin (units = the grid size).  zb = 2: a bin with an even z
// index and the next one (its z neighbour: nf[2] is even for these systems)
// share one window of 7 + P x 7 + P x 16 + P cells.  Each particle sums the
// same window cells in the same pairs either way (its offset in the window
// moves by 8 cells in z), so the results do not depend on zb.
template <typename T, int PT, bool FORCE>
__global__ void __launch_bounds__(I2_WARPS * 32, sizeof(T) == 4 ? 3 : 2) k_interp2(
    const SysDev* __restrict__ sys, const int* __restrict__ tab,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const int* __restrict__ sperm, const T* __restrict__ rows, const int* __restrict__ boff,
    const T* __restrict__ grid, double* __restrict__ out, double* __restrict__ phi_out,
    int Ep, int PL, int zb)
{
    using PV = Pair<T>;
    using VT = typename PV::V;
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ Interp2Warp<T> wsm[I2_WARPS];
    // the unit's system and first bin: two independent loads
    const int unit = blockIdx.x;
    const int bin = __ldg(tab + gridDim.x + unit);
    const int beg = boff[bin], end = boff[bin + zb];
    const SysDev& S = sys[__ldg(tab + unit)];
    const int lb = bin - S.bin_base;   // the unit's first bin in the system
    if (beg == end) return;
    const int P = PT ? PT : S.P;
    const int M = S.M;
    const int o0 = (lb / (S.nf[1] * S.nf[2])) * FB;
    const int o1 = ((lb / S.nf[2]) % S.nf[1]) * FB;
    const int o2 = (lb % S.nf[2]) * FB;
    const int E = FB + P - 1, EZ = interp2_ez(P, zb);
    T* tile = reinterpret_cast<T*>(dsm);
    const T* gs = grid + S.grid_off;
    const int warp = threadIdx.x >> 5;

    // ---- stage the window: rows (a, b), groups of 4 cells along z; thread t
    // copies group t % ng of rows t / ng, t / ng + R, ... (R rows per pass),
    // stepping (a, b) instead of dividing for every group
    {
        constexpr int G = 4;
        const int ng = EZ / G;
        const int R = blockDim.x / ng;
        const int g = threadIdx.x % ng, r0 = threadIdx.x / ng;
        const int Ra = R / E, Rb = R - Ra * E;
        int a = r0 / E, b = r0 - a * E;
        int z = o2 + g * G;
        z -= z >= M ? M : 0;
        const T* gz = gs + z;
        T* tz = tile + g * G;
        for (int row = r0 < R ? r0 : E * E; row < E * E; row += R) {
            int x = o0 + a, y = o1 + b;
            x -= x >= M ? M : 0;
            y -= y >= M ? M : 0;
            const T* src = gz + ((long long)x * M + y) * M;
            T* dst = tz + a * PL + b * Ep;
            a += Ra;
            b += Rb;
            if (b >= E) {
                b -= E;
                a++;
            }
#if SE_I2_ASYNC_STAGE
            // straight into shared memory: two copies of a cell pair each
            // (the window's rows are 8-byte aligned in FP32, 16 in FP64)
            if constexpr (sizeof(T) == 4) {
                cp_async8(dst, src);
                cp_async8(dst + 2, src + 2);
            } else {
                cp_async16(dst, src);
                cp_async16(dst + 2, src + 2);
            }
#else
            if constexpr (sizeof(T) == 4) {
                const float4 v = __ldg(reinterpret_cast<const float4*>(src));
                reinterpret_cast<float2*>(dst)[0] = make_float2(v.x, v.y);
                reinterpret_cast<float2*>(dst)[1] = make_float2(v.z, v.w);
            } else {
                const double2 v0 = __ldg(reinterpret_cast<const double2*>(src));
                const double2 v1 = __ldg(reinterpret_cast<const double2*>(src) + 1);
                reinterpret_cast<double2*>(dst)[0] = v0;
                reinterpret_cast<double2*>(dst)[1] = v1;
            }
#endif
        }
    }
#if SE_I2_ASYNC_STAGE
    cp_async_commit();
    cp_async_wait<0>();
#endif
    __syncthreads();

    Interp2Warp<T>& W = wsm[warp];
    const bool JFIX = (32 % P) == 0;
    if constexpr (sizeof(T) == 4) {
        // stencils whose P does not divide 32 (P = 12): x rows per lane; the
        // others keep the column mapping below, where each lane's y column is
        // fixed already (the choice depends on P alone, so a batch's
        // runtime-P kernel sums as the P-specialised one does)
        if (!JFIX) {
            interp2_rows_f32<PT, FORCE>(S, wsm[warp], reinterpret_cast<const float*>(tile), P,
                                        o0, o1, o2, beg + warp, end, srec, sg, sperm,
                                        reinterpret_cast<const float*>(rows), out, phi_out, Ep,
                                        PL);
        }
    }
    if (sizeof(T) == 4 && !JFIX) return;
    interp2_columns<T, PT, FORCE>(S, W, tile, P, o0, o1, o2, beg + warp, end, srec, sg, sperm,
                                  rows, out, phi_out, Ep, PL, JFIX);
}

// The column mapping (FP64, and FP32 with P dividing 32): lane l takes the
// (x, y) columns c = l, l + 32, ..., i = c / P, j = c % P.
template <typename T, int PT, bool FORCE>
__device__ __forceinline__ void interp2_columns(
    const SysDev& S, Interp2Warp<T>& W, const T* tile, int P, int o0, int o1, int o2,
    int pfirst, int pend, const double4* __restrict__ srec, const int* __restrict__ sg,
    const int* __restrict__ sperm, const T* __restrict__ rows, double* __restrict__ out,
    double* __restrict__ phi_out, int Ep, int PL, bool JFIX)
{
    using PV = Pair<T>;
    using VT = typename PV::V;
    const int lane = threadIdx.x & 31;
    constexpr bool force = FORCE;
    constexpr int NQ = PT ? PT / 2 + 1 : 9;   // z pairs a stencil spans (<= 9 for P <= 16)
    const int nq = P / 2 + 1;
    for (int p = pfirst; p < pend; p += I2_WARPS) {
        // the particle's three tile-aligned rows, entry l in lane l, loaded
        // beside its record: their addresses do not wait for the corner
        const T* rb = rows + (long long)p * 96;
        const T ex = rb[lane], ey = rb[32 + lane], ez = rb[64 + lane];
        const double4 rc = srec[p];
        const int pk = sg[p];
        const int orig = sperm[p];
        const int gx = g_of(pk, 0), gy = g_of(pk, 1), gz = g_of(pk, 2);
        const int r0 = gx - o0, r1 = gy - o1, r2 = gz - o2;
        // weights: lane i < P holds factor i of each axis, row entry
        // (g mod 16) + i (<= 30), from the lane that loaded it
        const T vx = __shfl_sync(0xffffffffu, ex, ((gx & 15) + lane) & 31);
        const T vy = __shfl_sync(0xffffffffu, ey, ((gy & 15) + lane) & 31);
        const T vz = __shfl_sync(0xffffffffu, ez, ((gz & 15) + lane) & 31);
        W.wz[lane] = T(0);
        W.fz[lane] = T(0);
        __syncwarp();
        if (lane < P) {
            const double off = (S.lo + lane) * S.h;
            W.wx[lane] = vx;
            W.wy[lane] = vy;
            W.wz[r2 + lane] = vz;
            if (force) {
                W.fx[lane] = (T)((double)vx * (-S.c * (rc.x - off)));
                W.fy[lane] = (T)((double)vy * (-S.c * (rc.y - off)));
                W.fz[r2 + lane] = (T)((double)vz * (-S.c * (rc.z - off)));
            }
        }
        __syncwarp();
        const int q0 = r2 >> 1;
        VT wz2[NQ], fz2[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            if (PT || q < nq) {
                wz2[q] = PV::load(W.wz + 2 * (q0 + q));
                fz2[q] = force ? PV::load(W.fz + 2 * (q0 + q)) : PV::zero();
            }
        }
        T a_pot = 0, a_fx = 0, a_fy = 0, a_fz = 0;
        // the columns, summing NQC z pairs each
        auto columns = [&](auto nqc) {
            constexpr int NQC = decltype(nqc)::value;
            if constexpr (PT != 0 && 32 % PT == 0) {
                // P divides 32: lane l's columns are rows i = l / P + m (32 / P)
                // of the fixed column j = l % P, m < P^2 / 32 -- the same
                // columns in the same order as the loop below, unrolled, with
                // the addresses a base and constant strides
                constexpr int STEP = 32 / PT, NCOL = PT * PT / 32;
                const int i0 = lane / PT, jl = lane % PT;
                const T* col0 = tile + (r0 + i0) * PL + (r1 + jl) * Ep + 2 * q0;
                const int cstep = STEP * PL;
#pragma unroll
                for (int m = 0; m < NCOL; m++) {
                    const T* col = col0 + m * cstep;
                    VT s0 = PV::zero(), s1 = PV::zero();
#pragma unroll
                    for (int q = 0; q < NQC; q++) {
                        const VT g2 = PV::load(col + 2 * q);
                        s0 = PV::fma(g2, wz2[q], s0);
                        if (force) s1 = PV::fma(g2, fz2[q], s1);
                    }
                    const T t0 = PV::sum(s0);
                    const T wxi = W.wx[i0 + m * STEP];
                    a_pot = fma(t0, wxi, a_pot);
                    if (force) {
                        a_fx = fma(t0, W.fx[i0 + m * STEP], a_fx);
                        a_fz = fma(PV::sum(s1), wxi, a_fz);
                    }
                }
            } else {
                for (int c = lane; c < P * P; c += 32) {
                    const int i = c / P, j = c - (c / P) * P;
                    const T* col = tile + (r0 + i) * PL + (r1 + j) * Ep + 2 * q0;
                    VT s0 = PV::zero(), s1 = PV::zero();
#pragma unroll
                    for (int q = 0; q < NQC; q++) {
                        if (PT || q < nq) {
                            const VT g2 = PV::load(col + 2 * q);
                            s0 = PV::fma(g2, wz2[q], s0);
                            if (force) s1 = PV::fma(g2, fz2[q], s1);
                        }
                    }
                    const T t0 = PV::sum(s0);
                    const T wxi = W.wx[i];
                    if (JFIX) {   // j is the lane's own: the y weights multiply once below
                        a_pot = fma(t0, wxi, a_pot);
                        if (force) {
                            a_fx = fma(t0, W.fx[i], a_fx);
                            a_fz = fma(PV::sum(s1), wxi, a_fz);
                        }
                    } else {
                        const T wyj = W.wy[j];
                        const T wij = wxi * wyj;
                        a_pot = fma(t0, wij, a_pot);
                        if (force) {
                            a_fx = fma(t0, W.fx[i] * wyj, a_fx);
                            a_fy = fma(t0, wxi * W.fy[j], a_fy);
                            a_fz = fma(PV::sum(s1), wij, a_fz);
                        }
                    }
                }
            }
        };
        // an even stencil that starts on a pair spans P/2 pairs, not P/2 + 1
        // (a warp-uniform choice: the pair the other form adds is zero)
        if (PT != 0 && PT % 2 == 0 && (r2 & 1) == 0)
            columns(std::integral_constant<int, (PT ? PT / 2 : 1)>{});
        else
            columns(std::integral_constant<int, NQ>{});
        double d_pot = a_pot, d_fx = a_fx, d_fy = a_fy, d_fz = a_fz;
        if (JFIX) {
            const int j = lane % P;
            const double wyj = (double)W.wy[j];
            if (force) {
                d_fy = d_pot * (double)W.fy[j];
                d_fx *= wyj;
                d_fz *= wyj;
            }
            d_pot *= wyj;
        }
        if (force && sizeof(T) == 4) {   // (the FP64 kernel has no registers to spare)
            warp_sum4(d_pot, d_fx, d_fy, d_fz);
        } else {
            d_pot = warp_sum(d_pot);
            if (force) {
                d_fx = warp_sum(d_fx);
                d_fy = warp_sum(d_fy);
                d_fz = warp_sum(d_fz);
            }
        }
        if (lane == 0)
            interp_store(S, orig - S.part_off, rc.w, d_pot, d_fx, d_fy, d_fz,
                         S.mode == SE_FORCE, out, phi_out);
        __syncwarp();
    }
}

// Every FP64 grid value of the batch as FP32 (the staged source of
// k_interp2<float>), two values per thread step.
// A thread converts CONVERT_ITEMS pairs a pass, loading them all first; the
// grid is at most CONVERT_CTAS CTAs of 256 (8 per SM of a B200).
constexpr int CONVERT_ITEMS = 4, CONVERT_CTAS = 148 * 8;

__global__ void k_grid_to_f32(const double2* __restrict__ in, float2* __restrict__ out,
                              long long n2)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; e0 < n2;
         e0 += stride * CONVERT_ITEMS) {
        double2 v[CONVERT_ITEMS];
#pragma unroll
        for (int k = 0; k < CONVERT_ITEMS; k++)
            if (e0 + k * stride < n2) v[k] = in[e0 + k * stride];
#pragma unroll
        for (int k = 0; k < CONVERT_ITEMS; k++)
            if (e0 + k * stride < n2) out[e0 + k * stride] = make_float2((float)v[k].x, (float)v[k].y);
    }
}
