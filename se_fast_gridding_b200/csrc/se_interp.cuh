// se_interp.cuh -- interpolation (SE_FGG_int / SE_FGG_int_force,
// SE_fgg.c:968-1100) with the periodic unfold (SE_FGG_extend_fcn,
// SE_fgg.c:417-443) fused.  Included inside namespace se by se_solve.cu.
//
// One CTA per fine bin (FB^3 stencil corners): the bin's window of
// E = FB + P - 1 cells per axis is staged from the periodic grid into shared
// memory (rows of the window are contiguous z runs of the grid; the periodic
// unfold is the index arithmetic), then one warp per particle gathers
//   phi = h^3 d sum_ijk H wx_i wy_j wz_k
//   F_a = h^3 d q sum_ijk H wx_i wy_j wz_k (-c u_a)      (SE_fgg.c:1083-1095)
// Lane l takes the (i, j) rows l, l+32, ...: the k sum of a row runs in the
// working precision against z factors held in registers, the row sums are
// combined in FP64 with per-row weights, and the warp reduces with shuffles.
//
// Shared-memory layout of the window: row pitch E|1 (odd) and a plane pitch
// chosen by the host so that the rows one warp reads at once fall in distinct
// banks.

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
struct InterpWarpSmem {
    double wx[MAX_P], wy[MAX_P];     // Gaussian factors, x and y
    double fx[MAX_P], fy[MAX_P];     // times -c u (force)
    __align__(16) T wz[MAX_P];       // z factors in the working precision
    __align__(16) T fz[MAX_P];
};

__device__ __forceinline__ void interp_store(const SysDev& S, int loc, double qw, double a_pot,
                                             double a_fx, double a_fy, double a_fz, bool force,
                                             double* __restrict__ out,
                                             double* __restrict__ phi_out)
{
    const double scale = S.h3 * S.d;
    if (force) {
        const double qs = qw / S.d * scale;   // q h^3 d
        out[S.out_off + loc] = qs * a_fx;
        out[S.out_off + loc + S.N] = qs * a_fy;
        out[S.out_off + loc + 2 * S.N] = qs * a_fz;
        if (phi_out) phi_out[S.part_off + loc] = scale * a_pot;
    } else {
        out[S.out_off + loc] = scale * a_pot;
    }
}

// One particle's factors (lane i < P holds factor i of each axis) into the
// warp's table, with the force factors w (-c u), u = t0 - (lo + i) h.
template <typename T>
__device__ __forceinline__ void set_factors(InterpWarpSmem<T>& W, const SysDev& S,
                                            const double4& rc, int P, int lane, T fx_, T fy_,
                                            T fz_)
{
    if (lane < P) {
        const double off = (S.lo + lane) * S.h;
        const double vx = (double)fx_, vy = (double)fy_, vz = (double)fz_;
        W.wx[lane] = vx;
        W.wy[lane] = vy;
        W.fx[lane] = vx * (-S.c * (rc.x - off));
        W.fy[lane] = vy * (-S.c * (rc.y - off));
        W.wz[lane] = (T)vz;
        W.fz[lane] = (T)(vz * (-S.c * (rc.z - off)));
    }
    __syncwarp();
}

// The same from the factor array (lanes < P load their own entries).
template <typename T>
__device__ __forceinline__ void load_factors(InterpWarpSmem<T>& W, const SysDev& S,
                                             const T* __restrict__ fac, int PS, long long p,
                                             const double4& rc, int P, int lane)
{
    const T* f = fac + p * 3 * PS;
    const bool in = lane < P;
    set_factors(W, S, rc, P, lane, in ? f[lane] : T(0), in ? f[PS + lane] : T(0),
                in ? f[2 * PS + lane] : T(0));
}

// PT = P at compile time (0: runtime P); plane = pitch between x planes of
// the staged window (elements).
template <typename T, int PT>
__global__ void __launch_bounds__(INTERP_WARPS * 32) k_interp(
    const SysDev* __restrict__ sys, const int* __restrict__ bin_prefix, int nsys,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const int* __restrict__ sperm, const T* __restrict__ fac, int PS,
    const T* __restrict__ rows, const int* __restrict__ boff, const double* __restrict__ grid,
    double* __restrict__ out, double* __restrict__ phi_out, int plane)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ InterpWarpSmem<T> wsm[INTERP_WARPS];
    const int bin = blockIdx.x;
    const int beg = boff[bin], end = boff[bin + 1];
    if (beg == end) return;
    const SysDev& S = sys[find_sys(bin_prefix, nsys, bin)];
    if (S.path & PATH_PAIR_INTERP) return;   // k_interp2 covers this system
    const int P = PT ? PT : S.P;
    const int M = S.M;
    const int lb = bin - S.bin_base;
    const int o0 = (lb / (S.nf[1] * S.nf[2])) * FB;
    const int o1 = ((lb / S.nf[2]) % S.nf[1]) * FB;
    const int o2 = (lb % S.nf[2]) * FB;
    const int E = FB + P - 1, Ep = E | 1;
    T* tile = reinterpret_cast<T*>(dsm);
    const double* gs = grid + S.grid_off;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // stage the periodic window [o, o + E) mod M: wrapped coordinates once per
    // axis, then a flat element loop (E is a compile-time constant for PT > 0)
    __shared__ int wrapped[3][FB + MAX_P];
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        wrapped[0][e] = pmod(o0 + e, M) * M;
        wrapped[1][e] = pmod(o1 + e, M);
        wrapped[2][e] = pmod(o2 + e, M);
    }
    __syncthreads();
    {
        constexpr int EC = FB + (PT ? PT : 1) - 1;
        const int EE = PT ? EC : E;
        for (int e = threadIdx.x; e < EE * EE * EE; e += blockDim.x) {
            const int a = e / (EE * EE), b = (e / EE) % EE, c = e % EE;
            tile[a * plane + b * Ep + c] =
                (T)gs[(long long)(wrapped[0][a] + wrapped[1][b]) * M + wrapped[2][c]];
        }
    }
    __syncthreads();
    InterpWarpSmem<T>& W = wsm[warp];
    const bool force = S.mode == SE_FORCE;
    // software pipeline: the next particle's record and factors are loaded
    // while the current one is summed
    double4 rc_n = make_double4(0, 0, 0, 0);
    int pk_n = 0, orig_n = 0;
    T vx_n = 0, vy_n = 0, vz_n = 0;
    auto fetch = [&](int q) {
        if (q < end) {
            rc_n = srec[q];
            pk_n = sg[q];
            orig_n = sperm[q];
            if (lane < P) {
                const T* f = fac + (long long)q * 3 * PS;
                vx_n = f[lane];
                vy_n = f[PS + lane];
                vz_n = f[2 * PS + lane];
            }
        }
    };
    fetch(beg + warp);
    for (int p = beg + warp; p < end; p += INTERP_WARPS) {
        const double4 rc = rc_n;
        const int pk = pk_n, orig = orig_n;
        const T vx = vx_n, vy = vy_n, vz = vz_n;
        fetch(p + INTERP_WARPS);
        const int r0 = g_of(pk, 0) - o0, r1 = g_of(pk, 1) - o1, r2 = g_of(pk, 2) - o2;
        set_factors(W, S, rc, P, lane, vx, vy, vz);
        constexpr int PR = PT ? PT : 1;
        T wz[PR], fz[PR];
        if (PT) {
#pragma unroll
            for (int k = 0; k < PR; k++) {
                wz[k] = W.wz[k];
                fz[k] = W.fz[k];
            }
        }
        // with 32 % P == 0 every row of a lane has the same j = lane % P (the
        // same test for compile-time and runtime P keeps the arithmetic, and so
        // the result, of a system identical alone and in a mixed batch)
        const bool JFIX = (32 % P) == 0;
        double a_pot = 0, a_fx = 0, a_fy = 0, a_fz = 0;
        for (int r = lane; r < P * P; r += 32) {
            const int i = r / P, j = r - (r / P) * P;
            const T* row = tile + (r0 + i) * plane + (r1 + j) * Ep + r2;
            T s0 = 0, s1 = 0;
            if (PT) {
#pragma unroll
                for (int k = 0; k < PR; k++) {
                    const T hv = row[k];
                    s0 = fma(hv, wz[k], s0);
                    if (force) s1 = fma(hv, fz[k], s1);
                }
            } else {
                for (int k = 0; k < P; k++) {
                    const T hv = row[k];
                    s0 = fma(hv, W.wz[k], s0);
                    if (force) s1 = fma(hv, W.fz[k], s1);
                }
            }
            const double d0 = (double)s0;
            if (JFIX) {   // j is the lane's own: the y weights multiply once below
                const double wxi = W.wx[i];
                a_pot = fma(d0, wxi, a_pot);
                if (force) {
                    a_fx = fma(d0, W.fx[i], a_fx);
                    a_fz = fma((double)s1, wxi, a_fz);
                }
            } else {
                const double wxi = W.wx[i], wyj = W.wy[j];
                a_pot = fma(d0, wxi * wyj, a_pot);
                if (force) {
                    a_fx = fma(d0, W.fx[i] * wyj, a_fx);
                    a_fy = fma(d0, wxi * W.fy[j], a_fy);
                    a_fz = fma((double)s1, wxi * wyj, a_fz);
                }
            }
        }
        if (JFIX) {
            const int j = lane % P;
            const double wyj = W.wy[j];
            if (force) {
                a_fy = a_pot * W.fy[j];
                a_fx *= wyj;
                a_fz *= wyj;
            }
            a_pot *= wyj;
        }
        a_pot = warp_sum(a_pot);
        if (force) {
            a_fx = warp_sum(a_fx);
            a_fy = warp_sum(a_fy);
            a_fz = warp_sum(a_fz);
        }
        if (lane == 0)
            interp_store(S, orig - S.part_off, rc.w, a_pot, a_fx, a_fy, a_fz, force, out,
                         phi_out);
        __syncwarp();
    }
}

// Interpolation without staging, for windows that exceed shared memory
// (large P): the same sums read from the periodic grid through L1/L2.
template <typename T>
__global__ void __launch_bounds__(INTERP_WARPS * 32) k_interp_global(
    const SysDev* __restrict__ sys, const int* __restrict__ part_prefix, int nsys, int ntot,
    const double4* __restrict__ srec, const int* __restrict__ sg,
    const int* __restrict__ sperm, const T* __restrict__ fac, int PS,
    const T* __restrict__ rows, const double* __restrict__ grid, double* __restrict__ out,
    double* __restrict__ phi_out)
{
    __shared__ InterpWarpSmem<T> wsm[INTERP_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * INTERP_WARPS + warp;
    if (p >= ntot) return;
    const int orig = sperm[p];
    const SysDev& S = sys[find_sys(part_prefix, nsys, orig)];
    if (S.path & PATH_PAIR_INTERP) return;   // k_interp2 covers this system
    const int P = S.P, M = S.M;
    InterpWarpSmem<T>& W = wsm[warp];
    const double4 rc = srec[p];
    const int pk = sg[p];
    const int g0 = g_of(pk, 0), g1 = g_of(pk, 1), g2 = g_of(pk, 2);
    load_factors(W, S, fac, PS, p, rc, P, lane);
    const bool force = S.mode == SE_FORCE;
    const double* gs = grid + S.grid_off;
    double a_pot = 0, a_fx = 0, a_fy = 0, a_fz = 0;
    for (int r = lane; r < P * P; r += 32) {
        const int i = r / P, j = r % P;
        const double* row = gs + ((long long)pmod(g0 + i, M) * M + pmod(g1 + j, M)) * M;
        double s0 = 0, s1 = 0;
        int z = g2;
        for (int k = 0; k < P; k++) {
            const double hv = __ldg(row + z);
            s0 = fma(hv, (double)W.wz[k], s0);
            if (force) s1 = fma(hv, (double)W.fz[k], s1);
            if (++z == M) z = 0;
        }
        const double wxi = W.wx[i], wyj = W.wy[j];
        a_pot = fma(s0, wxi * wyj, a_pot);
        if (force) {
            a_fx = fma(s0, W.fx[i] * wyj, a_fx);
            a_fy = fma(s0, wxi * W.fy[j], a_fy);
            a_fz = fma(s1, wxi * wyj, a_fz);
        }
    }
    a_pot = warp_sum(a_pot);
    if (force) {
        a_fx = warp_sum(a_fx);
        a_fy = warp_sum(a_fy);
        a_fz = warp_sum(a_fz);
    }
    if (lane == 0)
        interp_store(S, orig - S.part_off, rc.w, a_pot, a_fx, a_fy, a_fz, force, out, phi_out);
}
