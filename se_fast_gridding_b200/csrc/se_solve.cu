// se_solve.cu -- device-resident Spectral Ewald k-space solve on B200.
//
// One launch of each step covers every system of a batch (a single-system
// plan is a batch of one); per-system parameters and offsets live in a small
// device table (SysDev).
//
//   sort        per particle the stencil corner and offset as fgg_expansion_3p
//               (SE_fgg.c:539-621), charge x d and fine-bin key, then the
//               stable counting sort into bin order: k_bsort_count /
//               _columns / _scatter (se_binsort.cuh) for batches of at most
//               8192 bins and 2^19 particles, else k_prepare, the radix sort
//               of se_sort.cu and k_gather
//   k_factors   each particle's separable Gaussian factors, FGG recurrence
//               (tile-aligned rows for the tile kernels)
//   spread      k_tile_parts + k_spread2, one CTA per part of a 16^3 tile,
//               the fold fused (se_spread2.cuh), for grids of whole tiles and
//               P <= 16; k_spread (se_spread.cuh) for the others
//   cuFFT D2Z, k_scale (Z of scaling(), SE_general.c:145-175, applied to the
//               half spectrum as product_rc does, SE_general.c:336-362), Z2D
//   interp      k_grid_to_f32 (FP32 path) + k_interp2, one launch per stencil
//               of the batch, one CTA per fine bin or pair of z-adjacent bins
//               of its systems, the unfold fused (se_interp2.cuh), beside
//               k_spread2; k_interp (se_interp.cuh) for the others
//
// Grid layout: M^3 FP64 row-major [x][y][z], the transpose of the reference's
// column-major H_per; the FFT of the transpose is the transpose of the FFT and
// Z is symmetric in the axes, so results are identical.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "se_internal.h"

namespace se {

// --------------------------------------------------------------- errors ---

static thread_local char g_err_msg[256];

int cuda_fail(cudaError_t e, const char* what, const char* file, int line)
{
    snprintf(g_err_msg, sizeof(g_err_msg), "%s:%d %s: %s", file, line, what,
             cudaGetErrorString(e));
    fprintf(stderr, "[se_gpu] %s\n", g_err_msg);
    return e == cudaErrorMemoryAllocation ? SE_ERR_NOMEM : SE_ERR_CUDA;
}

static int cufft_fail(cufftResult r, const char* what)
{
    snprintf(g_err_msg, sizeof(g_err_msg), "cuFFT %s failed (%d)", what, (int)r);
    fprintf(stderr, "[se_gpu] %s\n", g_err_msg);
    return r == CUFFT_ALLOC_FAILED ? SE_ERR_NOMEM : SE_ERR_CUFFT;
}

#define SE_CUFFT(call)                                                        \
    do {                                                                      \
        cufftResult se_r_ = (call);                                           \
        if (se_r_ != CUFFT_SUCCESS) return cufft_fail(se_r_, #call);          \
    } while (0)

#include "se_device.cuh"

// --------------------------------------------------------------- prepare --

// Particle n (of system S, batch index) as the solve uses it: the stencil's
// first grid point per axis (wrapped into [0, M)), the offset t0 of the
// position from its nearest (odd P) or lower (even P) grid point, the charge
// times the spread constant, and the fine-bin key.  False for a NaN, infinite
// or absurd position: the particle then carries zero charge at cell 0.
__device__ __forceinline__ bool particle_of(const SysDev& S, const double* __restrict__ x,
                                            const double* __restrict__ q, int n, double4& rec,
                                            int& gpk, int& key)
{
    const int i = n - S.part_off;
    const double* xs = x + 3LL * S.part_off;
    const bool odd = S.P & 1;
    double t0[3];
    int g[3];
    bool ok = true;
    for (int a = 0; a < 3; a++) {
        const double xa = xs[i + (long long)a * S.N];
        const double u = xa / S.h;
        if (!(fabs(u) < 1.0e9)) {
            ok = false;
            t0[a] = 0.0;
            g[a] = 0;
            continue;
        }
        const int cell = odd ? (int)round(u) : (int)floor(u);
        t0[a] = __fma_rn(-S.h, (double)cell, xa);   // one rounding, in every kernel
        g[a] = pmod(cell + S.lo, S.M);
    }
    const double qw = ok ? q[n] * S.d : 0.0;
    rec = make_double4(t0[0], t0[1], t0[2], qw);
    gpk = pack_g(g[0], g[1], g[2]);
    key = S.bin_base + ((g[0] / FB) * S.nf[1] + g[1] / FB) * S.nf[2] + g[2] / FB;
    return ok;
}

__global__ void k_prepare(const SysDev* __restrict__ sys, const int* __restrict__ part_prefix,
                          int nsys, int ntot, const double* __restrict__ x,
                          const double* __restrict__ q, int* __restrict__ key,
                          double4* __restrict__ rec, int* __restrict__ gpk, int* err)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ntot) return;
    const SysDev& S = sys[find_sys(part_prefix, nsys, n)];
    double4 r;
    int g, k;
    if (!particle_of(S, x, q, n, r, g, k)) atomicOr(err, 1);
    rec[n] = r;
    gpk[n] = g;
    key[n] = k;
}

__global__ void k_gather(int ntot, const int* __restrict__ perm, const double4* __restrict__ rec,
                         const int* __restrict__ gpk, double4* __restrict__ srec,
                         int* __restrict__ sg)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ntot) return;
    const int j = perm[s];
    srec[s] = rec[j];
    sg[s] = gpk[j];
}

// The recurrence's first factor v0 = exp(-c u0^2) and ratio
// r0 = exp(2 c h u0 - c h^2), u0 = t0 - lo h, each operation rounded as
// written (no contraction), so every kernel that builds factors gets the
// same bits.
__device__ __forceinline__ void factor_start(const SysDev& S, double t0, double& v, double& r)
{
    const double u0 = __dsub_rn(t0, __dmul_rn(S.lo, S.h));
    v = exp(-__dmul_rn(__dmul_rn(S.c, u0), u0));
    const double ch = __dmul_rn(S.c, S.h);
    r = exp(__dsub_rn(__dmul_rn(__dmul_rn(2.0, ch), u0), __dmul_rn(ch, S.h)));
}

#include "se_binsort.cuh"

// ------------------------------------------------------- factor rows -----

// Each particle's separable Gaussian factors, once per solve, in bin order,
// built with the FGG recurrence in FP64 (SE_fgg.c:575-609 restated for the
// full Gaussian): v_0 = exp(-c u_0^2), r_0 = exp(2 c h u_0 - c h^2),
// v_{i+1} = v_i r_i, r_{i+1} = r_i exp(-2 c h^2), u_0 = t0 - lo h, stored in
// the working precision T.  Thread u = 3 s + a writes particle s, axis a:
//  - systems on a tile-aligned kernel (PATH_TILE_SPREAD / PATH_PAIR_INTERP): the tile-aligned 32-entry
//    row rows[u*32 + j] = f[j - (g_a mod 16)], zero outside the stencil; the
//    rows of a warp are contiguous, so they are staged in shared memory and
//    stored as one coalesced block;
//  - the others: fac[u*PS + i] = f[i], i < P (PS = the batch's largest P).
template <typename T>
constexpr int factors_threads() { return sizeof(T) == 4 ? 256 : 128; }

template <typename T>
__global__ void __launch_bounds__(factors_threads<T>()) k_factors(
    const SysDev* __restrict__ sys, const int* __restrict__ part_prefix, int nsys, int ntot,
    const double4* __restrict__ srec, const int* __restrict__ sperm, const int* __restrict__ sg,
    T* __restrict__ fac, int PS, T* __restrict__ rows)
{
    constexpr int V = 16 / sizeof(T);   // elements per 16 bytes
    constexpr int RS = 32 + V;          // staged row pitch, 16-byte aligned
    __shared__ __align__(16) T stage[factors_threads<T>()][RS];
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wbase = threadIdx.x & ~31;
    bool staged = false;
    if (u < 3 * ntot) {
        const int s = u / 3, a = u - 3 * (u / 3);
        const SysDev& S = sys[find_sys(part_prefix, nsys, sperm[s])];
        const double4 rc = srec[s];
        const double t0 = a == 0 ? rc.x : (a == 1 ? rc.y : rc.z);
        double v, r;
        factor_start(S, t0, v, r);
        const int tiled = S.path & (PATH_TILE_SPREAD | PATH_PAIR_INTERP);
        if (tiled) {
            staged = true;
            // a path that mixes tile-aligned and general kernels needs both rows
            T* f = tiled != (PATH_TILE_SPREAD | PATH_PAIR_INTERP) ? fac + (long long)u * PS
                                                                  : nullptr;
            T* st = stage[threadIdx.x];
#pragma unroll
            for (int j = 0; j < 32; j += V)
                *reinterpret_cast<uint4*>(st + j) = make_uint4(0u, 0u, 0u, 0u);
            st += ((unsigned)sg[s] >> (10 * a)) & 15u;
            for (int i = 0; i < S.P; i++) {
                st[i] = (T)v;
                if (f) f[i] = (T)v;
                v *= r;
                r *= S.rho;
            }
        } else {
            T* f = fac + (long long)u * PS;
            for (int i = 0; i < S.P; i++) {
                f[i] = (T)v;
                v *= r;
                r *= S.rho;
            }
        }
    }
    const unsigned srows = __ballot_sync(0xffffffffu, staged);
    if (!srows) return;
    __syncwarp();
    // the warp's 32 rows are rows[(u_w + k) * 32 ...], k < 32: one block
    const long long uw = (long long)blockIdx.x * blockDim.x + wbase;
    for (int k = lane; k < 32 * 32 / V; k += 32) {
        const int r = k / (32 / V), c = (k % (32 / V)) * V;
        if ((srows >> r) & 1u)
            *reinterpret_cast<uint4*>(rows + (uw + r) * 32 + c) =
                *reinterpret_cast<const uint4*>(&stage[wbase + r][c]);
    }
}

#include "se_spread.cuh"
#include "se_spread2.cuh"

// --------------------------------------------------------------- k-space --

__device__ __forceinline__ double kwave(int i, int M, double kfac)
{
    const int npos = (M % 2 == 0) ? M / 2 : (M - 1) / 2 + 1;
    return kfac * (double)(i < npos ? i : i - M);
}

// spec *= Z on the half spectrum [x][y][z <= M/2]; Z = exp(scalar K2)/K2 * 4pi/M^3
// with K2 summed in the reference's order (its first FFT axis is our z).
constexpr int SCALE_THREADS = 256, SCALE_ITEMS = 8;

// Elements e = blockIdx.x * SCALE_THREADS * SCALE_ITEMS + ... of the half
// spectrum [x][y][z <= M/2] of system order[first + blockIdx.y]; 32-bit
// index arithmetic.
__global__ void __launch_bounds__(SCALE_THREADS) k_scale(const SysDev* __restrict__ sys,
                                                         const int* __restrict__ order, int first,
                                                         double2* __restrict__ spec)
{
    const SysDev& S = sys[order[first + blockIdx.y]];
    const int M = S.M, Mh = M / 2 + 1;
    const int n = M * M * Mh;
    double2* sp = spec + S.spec_off;
    const int e0 = blockIdx.x * (SCALE_THREADS * SCALE_ITEMS) + threadIdx.x;
    // every load of the thread first, so they are in flight together
    double2 v[SCALE_ITEMS];
#pragma unroll
    for (int k = 0; k < SCALE_ITEMS; k++) {
        const int e = e0 + k * SCALE_THREADS;
        if (e < n) v[k] = sp[e];
    }
#pragma unroll
    for (int k = 0; k < SCALE_ITEMS; k++) {
        const int e = e0 + k * SCALE_THREADS;
        if (e >= n) break;
        const int r = e / Mh, iz = e - r * Mh;
        const int ix = r / M, iy = r - ix * M;
        const double kx = kwave(ix, M, S.kfac), ky = kwave(iy, M, S.kfac),
                     kz = kwave(iz, M, S.kfac);
        const double K2 = (kz * kz + ky * ky) + kx * kx;
        const double Z = (e == 0) ? 0.0 : exp(S.scalar * K2) / K2 * S.dnorm;
        v[k].x *= Z;
        v[k].y *= Z;
        sp[e] = v[k];
    }
}

// The same Z, computed in FP64, applied to an FP32 half spectrum.
__global__ void __launch_bounds__(SCALE_THREADS) k_scale32(const SysDev* __restrict__ sys,
                                                           float2* __restrict__ spec)
{
    const SysDev& S = sys[blockIdx.y];
    const int M = S.M, Mh = M / 2 + 1;
    const int n = M * M * Mh;
    float2* sp = spec + S.spec_off;
    const int e0 = blockIdx.x * (SCALE_THREADS * SCALE_ITEMS) + threadIdx.x;
    float2 v[SCALE_ITEMS];   // every load first, as in k_scale
#pragma unroll
    for (int k = 0; k < SCALE_ITEMS; k++) {
        const int e = e0 + k * SCALE_THREADS;
        if (e < n) v[k] = sp[e];
    }
#pragma unroll
    for (int k = 0; k < SCALE_ITEMS; k++) {
        const int e = e0 + k * SCALE_THREADS;
        if (e >= n) break;
        const int r = e / Mh, iz = e - r * Mh;
        const int ix = r / M, iy = r - ix * M;
        const double kx = kwave(ix, M, S.kfac), ky = kwave(iy, M, S.kfac),
                     kz = kwave(iz, M, S.kfac);
        const double K2 = (kz * kz + ky * ky) + kx * kx;
        const double Z = (e == 0) ? 0.0 : exp(S.scalar * K2) / K2 * S.dnorm;
        v[k].x = (float)((double)v[k].x * Z);
        v[k].y = (float)((double)v[k].y * Z);
        sp[e] = v[k];
    }
}

#include "se_fft.cuh"
#include "se_interp.cuh"
#include "se_interp2.cuh"

// FP32 grid back to FP64 (the FP32-FFT path feeding the general interpolation
// or a caller's FP64 grid).
__global__ void k_grid_to_f64(const float2* __restrict__ in, double2* __restrict__ out,
                              long long n2)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; e0 < n2;
         e0 += stride * CONVERT_ITEMS) {
        float2 v[CONVERT_ITEMS];
#pragma unroll
        for (int k = 0; k < CONVERT_ITEMS; k++)
            if (e0 + k * stride < n2) v[k] = in[e0 + k * stride];
#pragma unroll
        for (int k = 0; k < CONVERT_ITEMS; k++)
            if (e0 + k * stride < n2) out[e0 + k * stride] = make_double2((double)v[k].x, (double)v[k].y);
    }
}

// ---------------------------------------------------------------- energy --

__global__ void k_energy_partial(const double* __restrict__ phi, const double* __restrict__ q,
                                 int N, double* __restrict__ partial)
{
    __shared__ double ws[32];
    double s = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        s += phi[i] * q[i];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < blockDim.x / 32 ? ws[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

__global__ void k_energy_final(const double* __restrict__ partial, int n, double* e)
{
    __shared__ double ws[32];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < blockDim.x / 32 ? ws[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) *e = v / 2.;
    }
}

// ---------------------------------------------------------------- batch ---

struct HostSys {
    se_system d;
};

struct FftGroup {
    int M, count;
    int first;     // its systems are order[first .. first + count)
    bool custom;   // the three-pass FFT (se_fft.cuh), else cuFFT
    long long grid_off, spec_off;
    cufftHandle fwd, bwd;
};

// A captured solve and the arguments it was captured with.
struct GraphSlot {
    cudaGraphExec_t exec = nullptr;
    const void* key[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t stream = nullptr;
    int ntot = -1, launches = 0;
    bool timing = false;
    bool warm = false;   // the first solve with these arguments ran directly
};

}  // namespace se

struct se_batch_s {
    int nsys = 0, precision = SE_FP64;
    int ntot = 0, nbins = 0, ntiles = 0;
    long long grid_elems = 0, spec_elems = 0;
    std::vector<se::SysDev> host_sys;
    std::vector<int> part_prefix, tile_prefix, bin_prefix;
    std::vector<se::FftGroup> groups;
    // device
    se::SysDev* sys = nullptr;
    int* d_part_prefix = nullptr;
    int* d_tile_prefix = nullptr;
    int* d_bin_prefix = nullptr;
    int* key = nullptr;
    double4* rec = nullptr;
    int* gpk = nullptr;
    int* perm = nullptr;
    double4* srec = nullptr;
    int* sg = nullptr;
    int* boff = nullptr;
    void* fac = nullptr;      // per-particle factors [ntot][3][PS], working precision
    int PS = 0;
    void* rows = nullptr;     // tile-aligned rows [ntot][3][32] (k_spread2 systems)
    // k_spread2's split of crowded tiles: parts per tile (scanned), the
    // per-tile completion counters, the block counter of k_tile_parts, the
    // FP64 slabs of the parts after the first, and the launch bound
    int* tile_parts = nullptr;
    int* part_tile = nullptr;   // the tile of each part (written by k_tile_parts)
    int* tile_sys = nullptr;    // the system of each tile
    int* tile_done = nullptr;
    unsigned* tp_counter = nullptr;
    double* slab = nullptr;
    int slab_slots = 0;
    // k_spread2<float>'s CTAs per SM: S2_BLOCKS_FEW when every tile's CTA is
    // resident at once with 4 per SM (more registers, the same sums), else
    // S2_BLOCKS_MANY
    bool spread2_few = false;
    bool any_spread1 = false, any_spread2 = false;   // some system on k_spread / k_spread2
    bool any_interp1 = false, any_interp2 = false;   // on k_interp(_global) / k_interp2
    bool runtime_p = false;                          // some system asks for runtime P
    float* grid32 = nullptr;  // FP32 copy of the grids, staged by k_interp2<float>
    bool fft32 = false;       // SE_FP32_FFT32: FP32 FFTs on grid32 / spec32
    float2* spec32 = nullptr;
    // k_interp2 launches: one per stencil P of its systems (P-specialised
    // kernels where they exist), or one runtime-P launch over all of them
    // when some system asks for runtime P; each with its own window
    struct I2Class {
        int P = 0;              // the systems it serves (0: all, runtime P)
        int Pw = 0;             // the stencil its window is sized for
        bool special = false;   // the P-specialised kernel
        int Ep = 0, PL = 0;     // window pitches
        int zb = 1;             // z-adjacent bins per window (1 or 2)
        size_t smem = 0;
        int units = 0;          // CTAs: the systems' bins / zb
        int* tab = nullptr;     // device: each unit's system, then its first bin
    };
    std::vector<I2Class> i2_cls;
    bool i2_force = false;    // some k_interp2 system is in FORCE mode
    void* sort_scratch = nullptr;
    size_t sort_bytes = 0;
    bool bsort = false;   // the three-kernel bin sort (se_binsort.cuh) fits
    int* d_order = nullptr;      // system indices grouped by M (the FFT groups)
    double2* fft_tw = nullptr;   // W_128^k, k < 128, for the three-pass FFT
    double* grid = nullptr;
    double2* spec = nullptr;
    double* energy_partial = nullptr;
    int* err = nullptr;
    int launches = 0;
    int pending_launches = 0;   // issued before the next solve's own launches (rebind)
    int max_P = 0;
    bool staged_interp = true;
    size_t interp_smem = 0;
    int plane = 0;   // x-plane pitch of the staged interpolation window
    // per-stage CUDA events (prepare+sort, spread, k-space, interp)
    bool timing = false;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    // CUDA graphs of one solve: captured on the second solve with the same
    // buffers, stream and particle count, replayed after that.  Slot 0
    // serves the device-pointer entry points when se_*_set_graph turned it
    // on; slot 1 the host-buffer entry point, which owns its buffers and
    // stream and always replays.
    bool graph_on = false;
    se::GraphSlot gslot[2];
};

namespace se {

static void derive(int M, int P, double L, double xi, double m, double* h, double* w,
                   double* eta, double* c, double* d)
{
    // parse_params (SE_general.c:16-29), SE_FGG_FCN_params (SE_general.c:180-200)
    const double h0 = L / (double)M;
    const double w0 = (double)P * h0 / 2.;
    const double r = 2.0 * w0 * xi / m;
    const double eta0 = r * r;
    const double c0 = 2.0 * xi * xi / eta0;
    if (h) *h = L / M;
    if (w) *w = w0;
    if (eta) *eta = eta0;
    if (c) *c = c0;
    if (d) *d = pow(c0 / PI_D, 1.5);
}

static bool valid_system(const se_system& s)
{
    return s.N >= 0 && s.M >= 2 && s.M <= 1024 && s.P >= 1 && s.P <= MAX_P &&
           s.L > 0 && s.xi > 0 && s.m > 0 && (s.mode == SE_POTENTIAL || s.mode == SE_FORCE);
}

// The per-system fields of the device table that follow from (N, M, P, L,
// xi, m, mode): stencil offset, bin and tile counts, Gaussian and k-space
// constants.  Offsets into the batch's arrays are the caller's.
static void fill_sysdev(const se_system& s, SysDev& S)
{
    double h, w, eta, c, d;
    derive(s.M, s.P, s.L, s.xi, s.m, &h, &w, &eta, &c, &d);
    const int ph = (s.P & 1) ? (s.P - 1) / 2 : s.P / 2;
    S.N = s.N;
    S.M = s.M;
    S.P = s.P;
    S.lo = (s.P & 1) ? -ph : -ph + 1;
    S.mode = s.mode;
    S.path = default_path(s.M, s.P);
    const int nf = (s.M + FB - 1) / FB;
    S.nf[0] = S.nf[1] = S.nf[2] = nf;
    S.nt[0] = (s.M + TX - 1) / TX;
    S.nt[1] = (s.M + TY - 1) / TY;
    S.nt[2] = (s.M + TZ - 1) / TZ;
    S.h = h;
    S.c = c;
    S.d = d;
    S.h3 = h * h * h;
    S.rho = exp(-2.0 * c * h * h);
    S.kfac = 2.0 * PI_D / s.L;
    S.scalar = -(1. - eta) / (4. * s.xi * s.xi);
    S.dnorm = 4. * PI_D / (double)(s.M * s.M * s.M);
}

// Pitch between the x planes of the staged interpolation window: at least
// E * Ep, padded so that the rows one warp reads together (lane l takes row
// (l / P, l % P)) fall in as few 4-byte banks per wavefront as possible.
static int interp_plane(int P)
{
    const int E = FB + P - 1, Ep = E | 1;
    int best = E * Ep, best_conf = 1 << 30;
    for (int pad = 0; pad < 32; pad++) {
        const int plane = E * Ep + pad;
        int count[32] = {0};
        for (int l = 0; l < 32 && l < P * P; l++) {
            const int i = l / P, j = l % P;
            count[(i * plane + j * Ep) & 31]++;
        }
        int conf = 0;
        for (int b = 0; b < 32; b++) conf = std::max(conf, count[b]);
        if (conf < best_conf) {
            best_conf = conf;
            best = plane;
        }
    }
    return best;
}

static size_t interp_smem_bytes(int P, int precision)
{
    const int E = FB + P - 1;
    return (size_t)E * interp_plane(P) * (precision == SE_FP32 ? 4 : 8);
}

static int path_of(const se_system* sys, const int* paths, int i)
{
    return paths ? paths[i] : default_path(sys[i].M, sys[i].P);
}

// Slab slots k_spread2 may need for the particles of its systems: a bin is a
// candidate of at most 2 tiles per axis, so the candidates of all tiles sum
// to at most 8 N and the parts after each tile's first to 8 N / S2_CAP.
static int split_slots(long long ntile2)
{
    return (int)(8 * ntile2 / S2_CAP) + 1;
}

static size_t batch_bytes(const se_system* sys, int nsys, int precision, int* nbins_out,
                          int* ntiles_out, const int* paths = nullptr)
{
    const bool fft32 = precision == SE_FP32_FFT32;
    if (fft32) precision = SE_FP32;
    long long ntot = 0, nbins = 0, ntiles = 0, grid = 0, spec = 0;
    for (int i = 0; i < nsys; i++) {
        const int M = sys[i].M;
        const int nf = (M + FB - 1) / FB;
        ntot += sys[i].N;
        nbins += (long long)nf * nf * nf;
        ntiles += (long long)((M + TX - 1) / TX) * ((M + TY - 1) / TY) * ((M + TZ - 1) / TZ);
        grid += (long long)M * M * M + 16;
        spec += (long long)M * M * (M / 2 + 1);
    }
    if (nbins_out) *nbins_out = (int)nbins;
    if (ntiles_out) *ntiles_out = (int)ntiles;
    size_t b = 0;
    b += (size_t)ntot * (4 + 32 + 4 + 4 + 32 + 4);
    int maxP = 1;
    for (int i = 0; i < nsys; i++) maxP = std::max(maxP, sys[i].P);
    bool rows = false, plain = false, pair = false;
    for (int i = 0; i < nsys; i++) {
        const int t = path_of(sys, paths, i) & (PATH_TILE_SPREAD | PATH_PAIR_INTERP);
        if (t) rows = true;
        if (t != (PATH_TILE_SPREAD | PATH_PAIR_INTERP)) plain = true;
        if (t & PATH_PAIR_INTERP) pair = true;
    }
    if (plain) b += (size_t)ntot * 3 * maxP * (precision == SE_FP32 ? 4 : 8);
    if (rows) b += (size_t)ntot * 3 * 32 * (precision == SE_FP32 ? 4 : 8);
    long long ntile2 = 0;
    for (int i = 0; i < nsys; i++)
        if (path_of(sys, paths, i) & PATH_TILE_SPREAD) ntile2 += sys[i].N;
    if (ntile2 > 0 || rows)
        b += (size_t)split_slots(ntile2) * 4096 * 8 + (size_t)(2 * ntiles + 2) * 4;
    if ((pair && precision == SE_FP32) || fft32) b += (size_t)grid * 4;   // FP32 grids
    b += std::max(sort_scratch_bytes((int)ntot, (int)std::max<long long>(nbins, 1)),
                  bsort_scratch_bytes((int)std::max<long long>(nbins, 1)));
    b += (size_t)(nbins + 1) * 4;
    b += (size_t)grid * 8 + (size_t)spec * (fft32 ? 8 : 16);
    // cuFFT work areas are about one spectrum more
    b += (size_t)spec * (fft32 ? 8 : 16);
    b += (size_t)nsys * (sizeof(SysDev) + 12) + 4096;
    return b;
}

static void graph_drop(GraphSlot& g)
{
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    g.warm = false;
}

static void graph_drop(se_batch b)
{
    for (auto& g : b->gslot) graph_drop(g);
}

static int batch_free(se_batch b)
{
    if (!b) return SE_OK;
    graph_drop(b);
    for (auto& g : b->groups) {
        if (g.fwd) cufftDestroy(g.fwd);
        if (g.bwd) cufftDestroy(g.bwd);
    }
    for (auto& e : b->ev)
        if (e) cudaEventDestroy(e);
    for (auto& c : b->i2_cls)
        if (c.tab) cudaFree(c.tab);
    void* ptrs[] = {b->sys, b->d_part_prefix, b->d_tile_prefix, b->d_bin_prefix, b->key,
                    b->rec, b->gpk, b->perm, b->srec, b->sg, b->boff, b->sort_scratch,
                    b->grid, b->spec, b->energy_partial, b->err, b->fac, b->rows,
                    b->grid32, b->spec32, b->d_order, b->fft_tw, b->tile_parts,
                    b->tile_done, b->tp_counter, b->slab, b->part_tile, b->tile_sys};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete b;
    return SE_OK;
}

// The staged interpolation kernel a batch launches: specialised on P when
// every system has the same P in {8, 12, 16} (or 21 in FP64), else generic.
template <typename T>
static const void* staged_interp_variant(int P, bool uniform)
{
    if (uniform && P == 8) return (const void*)k_interp<T, 8>;
    if (uniform && P == 12) return (const void*)k_interp<T, 12>;
    if (uniform && P == 16) return (const void*)k_interp<T, 16>;
    if (sizeof(T) == 8 && uniform && P == 21) return (const void*)k_interp<T, 21>;
    return (const void*)k_interp<T, 0>;
}

static bool uniform_P(const se_batch_s* b)
{
    if (b->runtime_p) return false;   // the runtime-P variants were asked for
    for (auto& s : b->host_sys)
        if (s.P != b->max_P) return false;
    return true;
}

static const void* staged_interp_kernel(const se_batch_s* b)
{
    return b->precision == SE_FP32 ? staged_interp_variant<float>(b->max_P, uniform_P(b))
                                   : staged_interp_variant<double>(b->max_P, uniform_P(b));
}

// Dynamic shared memory a kernel may use is a per-device, per-function
// attribute shared by every plan in the process: only ever raise it, so a
// plan made later with a smaller window cannot break an earlier one.
static cudaError_t raise_smem_limit(const void* fn, size_t smem)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(mu);
    size_t& cur = limit[{dev, fn}];
    if (cur >= smem) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) cur = smem;
    return e;
}

// Row pitch Ep and plane pitch PL (elements, both even) of k_interp2's
// window of zb z-adjacent bins for stencils up to P: the pair loads of one
// warp instruction are served in 128-byte groups of lanes; count, over all
// load rounds m, the largest number of distinct 4-byte words that share a
// bank within a group, and keep the smallest among the windows of at most
// cap_bytes.  Returns false (and the smallest window) when none fits.
static bool interp2_pitch(int P, int precision, int zb, size_t cap_bytes, int* Ep_out,
                          int* PL_out)
{
    const int E = FB + P - 1, EZ = interp2_ez(P, zb);
    const size_t elem = precision == SE_FP32 ? 4 : 8;
    const int words = precision == SE_FP32 ? 2 : 4;   // 4-byte words per pair
    const int group = 32 / words;                     // lanes per 128 bytes
    // the lanes' (x, y) columns per load round: FP32 with P not dividing 32
    // (interp2_rows_f32) lane l takes row i = l % P and the columns
    // j = g J + m of its group g; otherwise lane l takes column c = l + 32 m,
    // i = c / P, j = c % P
    const int k = 32 / P, J = (P + k - 1) / k;
    const bool rows_map = precision == SE_FP32 && 32 % P != 0;
    const int rounds = rows_map ? J : (P * P + 31) / 32;
    auto column = [&](int l, int m, int* i, int* j) {
        if (rows_map) {
            const int g = std::min(l / P, k - 1);
            *i = l % P;
            *j = g * J + std::min(m, std::min(J, P - g * J) - 1);
            return true;
        }
        const int c = l + 32 * m;
        *i = c / P;
        *j = c % P;
        return c < P * P;
    };
    int best_cost = 1 << 30, best_Ep = EZ, best_PL = E * EZ;
    for (int Ep = EZ; Ep <= EZ + 32; Ep += 2) {
        for (int pad = 0; pad <= 64; pad += 2) {
            const int PL = E * Ep + pad;
            if ((size_t)E * PL * elem > cap_bytes) continue;
            int cost = 0;
            for (int m = 0; m < rounds; m++) {
                for (int g0 = 0; g0 < 32; g0 += group) {
                    int wordsat[32][8];
                    int nw[32] = {0};
                    int worst = 0;
                    for (int l = g0; l < g0 + group; l++) {
                        int ci, cj;
                        if (!column(l, m, &ci, &cj)) continue;
                        const int e = ci * PL + cj * Ep;   // element offset
                        for (int w = 0; w < words; w++) {
                            const int word = e * (words / 2) + w, bank = word & 31;
                            bool seen = false;
                            for (int k = 0; k < nw[bank]; k++) seen = seen || wordsat[bank][k] == word;
                            if (!seen && nw[bank] < 8) wordsat[bank][nw[bank]++] = word;
                            worst = std::max(worst, nw[bank]);
                        }
                    }
                    cost += worst;
                }
            }
            if (cost < best_cost) {
                best_cost = cost;
                best_Ep = Ep;
                best_PL = PL;
            }
        }
    }
    *Ep_out = best_Ep;
    *PL_out = best_PL;
    return best_cost < (1 << 30);
}

template <typename T, bool FORCE>
static const void* interp2_kernel(int P, bool special)
{
    return (special && P == 8)    ? (const void*)k_interp2<T, 8, FORCE>
           : (special && P == 12) ? (const void*)k_interp2<T, 12, FORCE>
           : (special && P == 16) ? (const void*)k_interp2<T, 16, FORCE>
                                  : (const void*)k_interp2<T, 0, FORCE>;
}

static bool interp2_special(int P) { return P == 8 || P == 12 || P == 16; }

// The k_interp2 window of a batch: two z-adjacent bins per window where the
// bins are sparse (at most I2_ZMERGE_MEAN particles per bin on average) and
// that window (beside the kernel's static shared memory) still leaves the
// CTAs per SM its launch bounds ask for (FP32: 3), else one bin.  Measured on
// B200: 100,000 particles in 4,096 bins (M = 128, P = 16) 0.139 -> 0.123 ms;
// 16M clustered particles in 262,144 bins (M = 512, P = 12) 11.3 -> 11.7 ms,
// where a window's copy is a small share of its particles' work and CTAs of
// two crowded bins lengthen the tail.
constexpr int I2_ZMERGE_MEAN = 32;
static int interp2_window(const se_batch_s* b, se_batch_s::I2Class& c, long long nparticles,
                          long long nbins, bool bin_windows)
{
    const bool fp32 = b->precision == SE_FP32;
    const bool force = b->i2_force;
    const void* fn = fp32 ? (force ? interp2_kernel<float, true>(c.Pw, c.special)
                                   : interp2_kernel<float, false>(c.Pw, c.special))
                          : (force ? interp2_kernel<double, true>(c.Pw, c.special)
                                   : interp2_kernel<double, false>(c.Pw, c.special));
    cudaFuncAttributes fa;
    SE_CUDA(cudaFuncGetAttributes(&fa, fn));
    int dev = 0, sm_bytes = 0, reserved = 0;
    SE_CUDA(cudaGetDevice(&dev));
    SE_CUDA(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    SE_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    const int ctas = fp32 ? 3 : 2;
    const long long cap = (long long)sm_bytes / ctas - reserved - (long long)fa.sharedSizeBytes;
    const size_t capb = cap > 0 ? (size_t)cap : 0;
    const bool sparse = nparticles <= (long long)I2_ZMERGE_MEAN * nbins;
    c.zb = 1;
    if (SE_I2_ZMERGE && fp32 && sparse && !bin_windows &&
        interp2_pitch(c.Pw, b->precision, 2, capb, &c.Ep, &c.PL))
        c.zb = 2;
    else   // one bin: the least conflicted pitch, whatever its size (the
           // pitch is worth more than a CTA per SM: FP64 P = 16 at the
           // smallest pitch that fits two CTAs ran 1.5x slower)
        interp2_pitch(c.Pw, b->precision, 1, (size_t)-1, &c.Ep, &c.PL);
    c.smem = (size_t)(FB + c.Pw - 1) * c.PL * (fp32 ? 4 : 8);
    return SE_OK;
}

// The units table of launch c (se_batch_s::I2Class::tab) for the systems
// `members`: every unit's system index, then every unit's first (global)
// bin, uploaded to the device.
static int interp2_table(se_batch_s* b, se_batch_s::I2Class& c, const std::vector<int>& members)
{
    std::vector<int> usys, ubin;
    for (int i : members) {
        const SysDev& S = b->host_sys[i];
        const int bins = S.nf[0] * S.nf[1] * S.nf[2];
        if (bins % c.zb) return SE_ERR_INVALID;   // zb = 2 needs pairs of z bins
        for (int lb = 0; lb < bins; lb += c.zb) {
            usys.push_back(i);
            ubin.push_back(S.bin_base + lb);
        }
    }
    c.units = (int)usys.size();
    std::vector<int> t(usys);
    t.insert(t.end(), ubin.begin(), ubin.end());
    if (t.empty()) return SE_OK;
    SE_CUDA(cudaMalloc(&c.tab, sizeof(int) * t.size()));
    SE_CUDA(cudaMemcpy(c.tab, t.data(), sizeof(int) * t.size(), cudaMemcpyHostToDevice));
    return SE_OK;
}

// The k_interp2 launches of a batch (se_batch_s::i2_cls).
static int interp2_classes(se_batch_s* b, const se_system* systems, int nsys)
{
    std::map<int, std::pair<long long, long long>> byP;   // P -> (particles, bins)
    bool bin_windows = false;
    int maxP = 0;
    long long np = 0, nb = 0;
    for (int i = 0; i < nsys; i++) {
        const SysDev& S = b->host_sys[i];
        if (!(S.path & PATH_PAIR_INTERP)) continue;
        const long long bins = (long long)S.nf[0] * S.nf[1] * S.nf[2];
        byP[systems[i].P].first += systems[i].N;
        byP[systems[i].P].second += bins;
        np += systems[i].N;
        nb += bins;
        maxP = std::max(maxP, systems[i].P);
        if (S.mode == SE_FORCE) b->i2_force = true;
        if (S.path & PATH_BIN_WINDOWS) bin_windows = true;
    }
    b->i2_cls.clear();
    auto members = [&](int P) {   // the pair-interpolation systems of stencil P (0: all)
        std::vector<int> v;
        for (int i = 0; i < nsys; i++)
            if ((b->host_sys[i].path & PATH_PAIR_INTERP) && (P == 0 || systems[i].P == P))
                v.push_back(i);
        return v;
    };
    if (b->runtime_p) {
        b->i2_cls.emplace_back();
        se_batch_s::I2Class& c = b->i2_cls.back();
        c.P = 0;
        c.Pw = maxP;
        SE_TRY(interp2_window(b, c, np, nb, bin_windows));
        return interp2_table(b, c, members(0));
    }
    for (const auto& kv : byP) {
        b->i2_cls.emplace_back();
        se_batch_s::I2Class& c = b->i2_cls.back();
        c.P = c.Pw = kv.first;
        c.special = interp2_special(kv.first);
        SE_TRY(interp2_window(b, c, kv.second.first, kv.second.second, bin_windows));
        SE_TRY(interp2_table(b, c, members(kv.first)));
    }
    return SE_OK;
}

static int batch_create(se_batch* out, const se_system* systems, int nsys, int precision,
                        const int* paths = nullptr)
{
    if (!out || !systems || nsys < 1 ||
        (precision != SE_FP64 && precision != SE_FP32 && precision != SE_FP32_FFT32))
        return SE_ERR_INVALID;
    const bool fft32 = precision == SE_FP32_FFT32;
    if (fft32) precision = SE_FP32;   // FP32 gridding; the FFTs in FP32 too
    for (int i = 0; i < nsys; i++) {
        if (!valid_system(systems[i])) return SE_ERR_INVALID;
        const int path = path_of(systems, paths, i);
        if (path < 0 || path > 63 ||
            ((path & (PATH_TILE_SPREAD | PATH_PAIR_INTERP)) &&
             !spread2_eligible(systems[i].M, systems[i].P)))
            return SE_ERR_INVALID;
    }
    se_batch b = new se_batch_s();
    b->nsys = nsys;
    b->precision = precision;
    b->fft32 = fft32;
    // grids grouped by M (batched FFT plans need contiguous equal sizes)
    std::vector<int> order(nsys);
    for (int i = 0; i < nsys; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return systems[a].M < systems[c].M; });
    std::vector<long long> goff(nsys), soff(nsys);
    long long gcur = 0, scur = 0;
    for (int k = 0; k < nsys; k++) {
        const int i = order[k];
        const int M = systems[i].M;
        if (b->groups.empty() || b->groups.back().M != M) {
            gcur = (gcur + 15) & ~15LL;   // every group's grids start 128-byte aligned
            FftGroup g{};
            g.M = M;
            g.count = 0;
            g.first = k;
            g.grid_off = gcur;
            g.spec_off = scur;
            b->groups.push_back(g);
        }
        b->groups.back().count++;
        goff[i] = gcur;
        soff[i] = scur;
        gcur += (long long)M * M * M;
        scur += (long long)M * M * (M / 2 + 1);
    }
    b->grid_elems = gcur;
    b->spec_elems = scur;
    int pcur = 0, ocur = 0, bcur = 0, tcur = 0;
    b->host_sys.resize(nsys);
    b->part_prefix.resize(nsys + 1);
    b->tile_prefix.resize(nsys + 1);
    b->bin_prefix.resize(nsys + 1);
    for (int i = 0; i < nsys; i++) {
        const se_system& s = systems[i];
        SysDev& S = b->host_sys[i];
        memset(&S, 0, sizeof(S));
        fill_sysdev(s, S);
        S.path = path_of(systems, paths, i);
        const int nf = S.nf[0];
        S.part_off = pcur;
        S.out_off = ocur;
        S.grid_off = goff[i];
        S.spec_off = soff[i];
        S.bin_base = bcur;
        S.tile_base = tcur;
        b->part_prefix[i] = pcur;
        b->tile_prefix[i] = tcur;
        b->bin_prefix[i] = bcur;
        pcur += s.N;
        ocur += (s.mode == SE_FORCE ? 3 : 1) * s.N;
        bcur += nf * nf * nf;
        tcur += S.nt[0] * S.nt[1] * S.nt[2];
        b->max_P = std::max(b->max_P, s.P);
    }
    b->part_prefix[nsys] = pcur;
    b->tile_prefix[nsys] = tcur;
    b->bin_prefix[nsys] = bcur;
    b->ntot = pcur;
    b->nbins = bcur;
    b->ntiles = tcur;
    {
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
            b->spread2_few = b->ntiles <= S2_BLOCKS_FEW * sms;
    }
    b->interp_smem = interp_smem_bytes(b->max_P, precision);
    b->plane = interp_plane(b->max_P);
    b->staged_interp = b->interp_smem + sizeof(InterpWarpSmem<double>) * INTERP_WARPS <= 220 * 1024;

    auto fail = [&](int code) {
        batch_free(b);
        return code;
    };
#define SE_ALLOC(ptr, bytes)                                                    \
    do {                                                                        \
        cudaError_t e_ = cudaMalloc((void**)&(ptr), std::max<size_t>((bytes), 16)); \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, "cudaMalloc", __FILE__, __LINE__)); \
    } while (0)
    const size_t nt = (size_t)std::max(b->ntot, 1);
    SE_ALLOC(b->sys, sizeof(SysDev) * nsys);
    SE_ALLOC(b->d_part_prefix, sizeof(int) * (nsys + 1));
    SE_ALLOC(b->d_tile_prefix, sizeof(int) * (nsys + 1));
    SE_ALLOC(b->d_bin_prefix, sizeof(int) * (nsys + 1));
    SE_ALLOC(b->key, sizeof(int) * nt);
    SE_ALLOC(b->rec, sizeof(double4) * nt);
    SE_ALLOC(b->gpk, sizeof(int) * nt);
    SE_ALLOC(b->perm, sizeof(int) * nt);
    SE_ALLOC(b->srec, sizeof(double4) * nt);
    SE_ALLOC(b->sg, sizeof(int) * nt);
    SE_ALLOC(b->boff, sizeof(int) * (b->nbins + 1));
    b->PS = b->max_P;
    bool need_fac = false, need_rows = false;
    for (int i = 0; i < nsys; i++) {
        const int path = b->host_sys[i].path;
        (path & PATH_TILE_SPREAD ? b->any_spread2 : b->any_spread1) = true;
        (path & PATH_PAIR_INTERP ? b->any_interp2 : b->any_interp1) = true;
        if (path & PATH_RUNTIME_P) b->runtime_p = true;
        const int t = path & (PATH_TILE_SPREAD | PATH_PAIR_INTERP);
        if (t) need_rows = true;
        if (t != (PATH_TILE_SPREAD | PATH_PAIR_INTERP)) need_fac = true;
    }
    if (need_fac) SE_ALLOC(b->fac, nt * 3 * b->PS * (precision == SE_FP32 ? 4 : 8));
    if (need_rows) SE_ALLOC(b->rows, nt * 3 * 32 * (precision == SE_FP32 ? 4 : 8));
    if (b->any_spread2) {
        long long ntile2 = 0;
        for (int i = 0; i < nsys; i++)
            if (b->host_sys[i].path & PATH_TILE_SPREAD) ntile2 += systems[i].N;
        b->slab_slots = split_slots(ntile2);
        SE_ALLOC(b->tile_parts, sizeof(int) * (b->ntiles + 1));
        SE_ALLOC(b->part_tile, sizeof(int) * (size_t)(b->ntiles + b->slab_slots));
        SE_ALLOC(b->tile_sys, sizeof(int) * std::max(b->ntiles, 1));
        {   // every entry a valid tile from the start (k_tile_parts rewrites them per solve)
            const cudaError_t z = cudaMemset(b->part_tile, 0, sizeof(int) * (size_t)(b->ntiles + b->slab_slots));
            if (z != cudaSuccess) return fail(cuda_fail(z, "cudaMemset", __FILE__, __LINE__));
        }
        SE_ALLOC(b->tile_done, sizeof(int) * std::max(b->ntiles, 1));
        SE_ALLOC(b->tp_counter, sizeof(unsigned));
        SE_ALLOC(b->slab, sizeof(double) * 4096 * (size_t)b->slab_slots);
    }
    if ((b->any_interp2 && precision == SE_FP32) || fft32)
        SE_ALLOC(b->grid32, sizeof(float) * (b->grid_elems + 16));
    if (fft32) SE_ALLOC(b->spec32, sizeof(float2) * b->spec_elems);
    if (b->any_interp2) {
        const int rc = interp2_classes(b, systems, nsys);
        if (rc != SE_OK) return fail(rc);
    }
    b->bsort = bsort_fits(b->ntot, b->nbins);
    for (int i = 0; i < nsys; i++)
        if (b->host_sys[i].path & PATH_RADIX_SORT) b->bsort = false;
    b->sort_bytes = std::max(sort_scratch_bytes(b->ntot, std::max(b->nbins, 1)),
                             b->bsort ? bsort_scratch_bytes(b->nbins) : size_t(0));
    SE_ALLOC(b->sort_scratch, b->sort_bytes);
    SE_ALLOC(b->grid, sizeof(double) * (b->grid_elems + 16));
    if (!fft32) SE_ALLOC(b->spec, sizeof(double2) * b->spec_elems);
    SE_ALLOC(b->energy_partial, sizeof(double) * 1024);
    SE_ALLOC(b->err, sizeof(int));
    SE_ALLOC(b->d_order, sizeof(int) * nsys);
    SE_ALLOC(b->fft_tw, sizeof(double2) * 128);
#undef SE_ALLOC
    cudaError_t e = cudaMemcpy(b->sys, b->host_sys.data(), sizeof(SysDev) * nsys,
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_part_prefix, b->part_prefix.data(), sizeof(int) * (nsys + 1),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_tile_prefix, b->tile_prefix.data(), sizeof(int) * (nsys + 1),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_bin_prefix, b->bin_prefix.data(), sizeof(int) * (nsys + 1),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess && b->tile_sys) {
        std::vector<int> ts(std::max(b->ntiles, 1), 0);
        for (int i = 0; i < nsys; i++)
            for (int t = b->tile_prefix[i]; t < b->tile_prefix[i + 1]; t++) ts[t] = i;
        e = cudaMemcpy(b->tile_sys, ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(b->err, 0, sizeof(int));
    if (e == cudaSuccess && b->tile_done)
        e = cudaMemset(b->tile_done, 0, sizeof(int) * std::max(b->ntiles, 1));
    if (e == cudaSuccess && b->tp_counter) e = cudaMemset(b->tp_counter, 0, sizeof(unsigned));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_order, order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        // W_128^k = exp(-2 pi i k / 128), rounded once from long double
        double2 tw[128];
        const long double two_pi = 6.283185307179586476925286766559005768L;
        for (int k = 0; k < 128; k++) {
            const long double a = two_pi * (long double)k / 128.0L;
            tw[k] = make_double2((double)cosl(a), (double)-sinl(a));
        }
        e = cudaMemcpy(b->fft_tw, tw, sizeof(tw), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMemcpy", __FILE__, __LINE__));
    // on request, the three-pass FFT takes the FP64 transforms of M = 32, 64, 128
    bool fft3 = false;
    for (int i = 0; i < nsys; i++)
        if (b->host_sys[i].path & PATH_FFT3) fft3 = !fft32;
    for (auto& g : b->groups) g.custom = fft3 && (g.M == 32 || g.M == 64 || g.M == 128);
    for (auto& g : b->groups) {
        if (g.custom) continue;
        int n[3] = {g.M, g.M, g.M};
        const int idist = g.M * g.M * g.M, odist = g.M * g.M * (g.M / 2 + 1);
        cufftResult r = cufftPlanMany(&g.fwd, 3, n, nullptr, 1, idist, nullptr, 1, odist,
                                      fft32 ? CUFFT_R2C : CUFFT_D2Z, g.count);
        if (r == CUFFT_SUCCESS)
            r = cufftPlanMany(&g.bwd, 3, n, nullptr, 1, odist, nullptr, 1, idist,
                              fft32 ? CUFFT_C2R : CUFFT_Z2D, g.count);
        if (r != CUFFT_SUCCESS) return fail(cufft_fail(r, "cufftPlanMany"));
    }
    {
        // the spread tiles want up to five CTAs of ~43 KB shared memory per SM
        const int carve = (int)cudaSharedmemCarveoutMaxShared;
        cudaError_t a = cudaFuncSetAttribute((const void*)k_spread<float>,
                                             cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        if (a == cudaSuccess)
            a = cudaFuncSetAttribute((const void*)k_spread<double>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        if (a == cudaSuccess)
            a = cudaFuncSetAttribute((const void*)k_spread2<float, S2_BLOCKS_MANY>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        if (a == cudaSuccess)
            a = cudaFuncSetAttribute((const void*)k_spread2<float, S2_BLOCKS_FEW>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        if (a == cudaSuccess)
            a = cudaFuncSetAttribute((const void*)k_spread2<float, S2_BLOCKS_MANY, 1>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        if (a == cudaSuccess)
            a = cudaFuncSetAttribute((const void*)k_spread2<double, S2_BLOCKS_FP64>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        if (a != cudaSuccess) return fail(cuda_fail(a, "cudaFuncSetAttribute", __FILE__, __LINE__));
    }
    if (b->staged_interp) {
        const cudaError_t a = raise_smem_limit(staged_interp_kernel(b), b->interp_smem);
        if (a != cudaSuccess) return fail(cuda_fail(a, "cudaFuncSetAttribute", __FILE__, __LINE__));
    }
    for (const auto& g : b->groups) {
        if (!g.custom) continue;
        cudaError_t a = cudaSuccess;
        if (g.M == 128) {
            a = raise_smem_limit((const void*)k_fft_zy<128>, fft_plane_smem<128>());
            if (a == cudaSuccess) a = raise_smem_limit((const void*)k_ifft_yz<128>, fft_plane_smem<128>());
        }
        if (a != cudaSuccess) return fail(cuda_fail(a, "cudaFuncSetAttribute", __FILE__, __LINE__));
    }
    *out = b;
    return SE_OK;
}

#define LAUNCHED(b) ((b)->launches++)

static int run_factors(se_batch b, cudaStream_t st);

static int run_bin_sort(se_batch b, const double* x, const double* q, cudaStream_t st)
{
    const int nk = b->nbins, chunk = bsort_chunk(b->ntot);
    const int nch = ceil_div(b->ntot, chunk);
    int* H = static_cast<int*>(b->sort_scratch);
    int* T = H + (size_t)BSORT_MAX_CHUNKS * nk;
    k_bsort_count<<<nch, BSORT_THREADS, sizeof(int) * nk, st>>>(
        b->sys, b->d_part_prefix, b->nsys, b->ntot, x, q, chunk, nk, b->key, H, b->err);
    SE_CUDA(cudaGetLastError());
    k_bsort_columns<<<ceil_div(nk, 32), BSORT_COL_WARPS * 32, 0, st>>>(H, nch, nk, T);
    SE_CUDA(cudaGetLastError());
    const size_t smem = bsort_scatter_smem(b->ntot, nk);
    SE_CUDA(raise_smem_limit((const void*)k_bsort_scatter, smem));
    k_bsort_scatter<<<nch, BSORT_THREADS, smem, st>>>(b->sys, b->d_part_prefix, b->nsys,
                                                      b->ntot, x, q, chunk, nk, b->key, H, T,
                                                      b->boff, b->perm, b->srec, b->sg, b->err);
    SE_CUDA(cudaGetLastError());
    b->launches += 3;
    return run_factors(b, st);
}

static int run_prepare_sort(se_batch b, const double* x, const double* q, cudaStream_t st)
{
    if (b->bsort && b->ntot > 0) return run_bin_sort(b, x, q, st);
    if (b->ntot > 0) {
        k_prepare<<<ceil_div(b->ntot, 256), 256, 0, st>>>(b->sys, b->d_part_prefix, b->nsys,
                                                          b->ntot, x, q, b->key, b->rec,
                                                          b->gpk, b->err);
        SE_CUDA(cudaGetLastError());
        LAUNCHED(b);
    }
    SE_TRY(stable_sort(b->key, nullptr, b->ntot, std::max(b->nbins, 1), b->perm, nullptr,
                       b->boff, b->sort_scratch, b->sort_bytes, st, &b->launches));
    if (b->ntot > 0) {
        k_gather<<<ceil_div(b->ntot, 256), 256, 0, st>>>(b->ntot, b->perm, b->rec, b->gpk,
                                                         b->srec, b->sg);
        SE_CUDA(cudaGetLastError());
        LAUNCHED(b);
    }
    return run_factors(b, st);
}

static int run_spread(se_batch b, double* grid, cudaStream_t st)
{
    // every tile is written by exactly one of the two kernels (by system)
    if (b->any_spread2) {
        // the parts of each tile and each part's tile, then one CTA per part
        // (at most the bound; the CTAs past the number of parts return at once)
        const int bound = b->ntiles + b->slab_slots;
        k_tile_parts<<<ceil_div(b->ntiles, TP_TILES), TP_WARPS * 32, 0, st>>>(
            b->sys, b->d_tile_prefix, b->nsys, b->ntiles, b->boff, b->tile_parts, b->tp_counter,
            bound, b->err, b->part_tile);
        SE_CUDA(cudaGetLastError());
        LAUNCHED(b);
        constexpr int SPLIT = S2_WARPS / S2_CTA_WARPS;
        if (b->precision == SE_FP32 && !b->spread2_few && b->ntiles >= S2_ONE_WARP_TILES)
            k_spread2<float, S2_BLOCKS_MANY, 1><<<bound * S2_WARPS, 32, 0, st>>>(
                b->sys, b->tile_sys, b->srec, b->sg, static_cast<const float*>(b->rows), b->boff,
                grid, b->tile_parts, b->part_tile, b->ntiles, b->tile_done, b->slab,
                b->slab_slots, b->err);
        else if (b->precision == SE_FP32)
            (b->spread2_few ? k_spread2<float, S2_BLOCKS_FEW> : k_spread2<float, S2_BLOCKS_MANY>)
                <<<bound * SPLIT, S2_CTA_WARPS * 32, 0, st>>>(
                    b->sys, b->tile_sys, b->srec, b->sg,
                    static_cast<const float*>(b->rows), b->boff, grid, b->tile_parts,
                    b->part_tile, b->ntiles,
                    b->tile_done, b->slab, b->slab_slots, b->err);
        else
            k_spread2<double, S2_BLOCKS_FP64><<<bound * SPLIT, S2_CTA_WARPS * 32, 0, st>>>(
                b->sys, b->tile_sys, b->srec, b->sg,
                static_cast<const double*>(b->rows), b->boff, grid, b->tile_parts,
                b->part_tile, b->ntiles,
                b->tile_done, b->slab, b->slab_slots, b->err);
        SE_CUDA(cudaGetLastError());
        LAUNCHED(b);
    }
    if (b->any_spread1) {
        if (b->precision == SE_FP32)
            k_spread<float><<<b->ntiles, SPREAD_THREADS, 0, st>>>(
                b->sys, b->d_tile_prefix, b->nsys, b->srec, b->sg,
                static_cast<const float*>(b->fac), b->PS, b->boff, grid);
        else
            k_spread<double><<<b->ntiles, SPREAD_THREADS, 0, st>>>(
                b->sys, b->d_tile_prefix, b->nsys, b->srec, b->sg,
                static_cast<const double*>(b->fac), b->PS, b->boff, grid);
        SE_CUDA(cudaGetLastError());
        LAUNCHED(b);
    }
    return SE_OK;
}

// FP64 <-> FP32 copies of the batch's grids (pairs; the allocations carry
// one spare element so an odd total is covered).
static int grid_f64_to_f32(se_batch b, const double* grid, cudaStream_t st)
{
    const long long n2 = (b->grid_elems + 1) / 2;
    k_grid_to_f32<<<std::min<long long>(CONVERT_CTAS, ceil_div(n2, 256 * CONVERT_ITEMS)), 256, 0, st>>>(
        reinterpret_cast<const double2*>(grid), reinterpret_cast<float2*>(b->grid32), n2);
    SE_CUDA(cudaGetLastError());
    LAUNCHED(b);
    return SE_OK;
}

static int grid_f32_to_f64(se_batch b, double* grid, cudaStream_t st)
{
    const long long n2 = (b->grid_elems + 1) / 2;
    k_grid_to_f64<<<std::min<long long>(CONVERT_CTAS, ceil_div(n2, 256 * CONVERT_ITEMS)), 256, 0, st>>>(
        reinterpret_cast<const float2*>(b->grid32), reinterpret_cast<double2*>(grid), n2);
    SE_CUDA(cudaGetLastError());
    LAUNCHED(b);
    return SE_OK;
}

// SE_FP32_FFT32: the grid to FP32, R2C, Z (computed in FP64) on the FP32
// half spectrum, C2R; the result stays in grid32.
static int run_kspace32(se_batch b, const double* grid, cudaStream_t st)
{
    SE_TRY(grid_f64_to_f32(b, grid, st));
    for (auto& g : b->groups) {
        SE_CUFFT(cufftSetStream(g.fwd, st));
        SE_CUFFT(cufftExecR2C(g.fwd, b->grid32 + g.grid_off,
                              reinterpret_cast<cufftComplex*>(b->spec32 + g.spec_off)));
    }
    int maxM = 0;
    for (auto& g : b->groups) maxM = std::max(maxM, g.M);
    const dim3 gs(ceil_div((long)maxM * maxM * (maxM / 2 + 1), SCALE_THREADS * SCALE_ITEMS),
                  b->nsys);
    k_scale32<<<gs, SCALE_THREADS, 0, st>>>(b->sys, b->spec32);
    SE_CUDA(cudaGetLastError());
    LAUNCHED(b);
    for (auto& g : b->groups) {
        SE_CUFFT(cufftSetStream(g.bwd, st));
        SE_CUFFT(cufftExecC2R(g.bwd, reinterpret_cast<cufftComplex*>(b->spec32 + g.spec_off),
                              b->grid32 + g.grid_off));
    }
    return SE_OK;
}

// The three passes of se_fft.cuh for group g; grid32 (may be null) receives
// the FP32 copy of the result beside the FP64 grid.
template <int M>
static int launch_fft3(se_batch b, const FftGroup& g, double* grid, float* grid32, cudaStream_t st)
{
    const unsigned planes = (unsigned)(g.count * M);
    k_fft_zy<M><<<planes, FFT_THREADS, fft_plane_smem<M>(), st>>>(b->sys, b->d_order, g.first,
                                                                  grid, b->spec, b->fft_tw);
    SE_CUDA(cudaGetLastError());
    k_fft_x_scale<M><<<(unsigned)(g.count * M * fft_x_blocks<M>()), FFT_X_THREADS, 0, st>>>(
        b->sys, b->d_order, g.first, b->spec, b->fft_tw);
    SE_CUDA(cudaGetLastError());
    k_ifft_yz<M><<<planes, FFT_THREADS, fft_plane_smem<M>(), st>>>(
        b->sys, b->d_order, g.first, b->spec, grid, grid32, b->fft_tw);
    SE_CUDA(cudaGetLastError());
    b->launches += 3;
    return SE_OK;
}

// grid32_fresh (may be null): set when every group's result was also
// written to the FP32 grids.
static int run_kspace(se_batch b, double* grid, cudaStream_t st, bool* grid32_fresh = nullptr)
{
    if (grid32_fresh) *grid32_fresh = false;
    if (b->fft32) return run_kspace32(b, grid, st);
    bool all_custom = true;
    for (const auto& g : b->groups) all_custom = all_custom && g.custom;
    float* g32 = (all_custom && b->grid32) ? b->grid32 : nullptr;
    for (const auto& g : b->groups) {
        if (!g.custom) continue;
        // the kernels add each system's own grid offset to the batch's bases
        if (g.M == 128) SE_TRY(launch_fft3<128>(b, g, grid, g32, st));
        else if (g.M == 64) SE_TRY(launch_fft3<64>(b, g, grid, g32, st));
        else SE_TRY(launch_fft3<32>(b, g, grid, g32, st));
    }
    if (grid32_fresh) *grid32_fresh = g32 != nullptr;
    for (const auto& g : b->groups) {
        if (g.custom) continue;
        SE_CUFFT(cufftSetStream(g.fwd, st));
        SE_CUFFT(cufftExecD2Z(g.fwd, grid + g.grid_off,
                              reinterpret_cast<cufftDoubleComplex*>(b->spec + g.spec_off)));
        const dim3 gs(ceil_div((long)g.M * g.M * (g.M / 2 + 1), SCALE_THREADS * SCALE_ITEMS),
                      g.count);
        k_scale<<<gs, SCALE_THREADS, 0, st>>>(b->sys, b->d_order, g.first, b->spec);
        SE_CUDA(cudaGetLastError());
        LAUNCHED(b);
        SE_CUFFT(cufftSetStream(g.bwd, st));
        SE_CUFFT(cufftExecZ2D(g.bwd,
                              reinterpret_cast<cufftDoubleComplex*>(b->spec + g.spec_off),
                              grid + g.grid_off));
    }
    return SE_OK;
}

template <typename T>
static int launch_interp_staged(se_batch b, const double* grid, double* out, double* phi,
                                cudaStream_t st)
{
    const size_t smem = b->interp_smem;
    const int P = b->max_P;
    const bool uniform = uniform_P(b);
    const dim3 grd(std::max(b->nbins, 1)), blk(INTERP_WARPS * 32);
    const T* fac = static_cast<const T*>(b->fac);
    const T* rows = static_cast<const T*>(b->rows);
#define SE_IARGS b->sys, b->d_bin_prefix, b->nsys, b->srec, b->sg, b->perm, fac, b->PS, rows, \
                 b->boff, grid, out, phi, b->plane
    if (uniform && P == 8) k_interp<T, 8><<<grd, blk, smem, st>>>(SE_IARGS);
    else if (uniform && P == 12) k_interp<T, 12><<<grd, blk, smem, st>>>(SE_IARGS);
    else if (uniform && P == 16) k_interp<T, 16><<<grd, blk, smem, st>>>(SE_IARGS);
    else if (sizeof(T) == 8 && uniform && P == 21) k_interp<T, 21><<<grd, blk, smem, st>>>(SE_IARGS);
    else k_interp<T, 0><<<grd, blk, smem, st>>>(SE_IARGS);
#undef SE_IARGS
    SE_CUDA(cudaGetLastError());
    LAUNCHED(b);
    return SE_OK;
}

static int run_factors(se_batch b, cudaStream_t st)
{
    if (b->ntot == 0) return SE_OK;
    if (b->precision == SE_FP32)
        k_factors<float><<<ceil_div(3L * b->ntot, factors_threads<float>()),
                           factors_threads<float>(), 0, st>>>(
            b->sys, b->d_part_prefix, b->nsys, b->ntot, b->srec, b->perm, b->sg,
            static_cast<float*>(b->fac), b->PS, static_cast<float*>(b->rows));
    else
        k_factors<double><<<ceil_div(3L * b->ntot, factors_threads<double>()),
                            factors_threads<double>(), 0, st>>>(
            b->sys, b->d_part_prefix, b->nsys, b->ntot, b->srec, b->perm, b->sg,
            static_cast<double*>(b->fac), b->PS, static_cast<double*>(b->rows));
    SE_CUDA(cudaGetLastError());
    LAUNCHED(b);
    return SE_OK;
}

template <typename T, bool FORCE>
static int launch_interp2_mode(se_batch b, const T* grid, double* out, double* phi,
                               cudaStream_t st)
{
    // one launch per class, one CTA per unit of its systems' bins
    const dim3 blk(I2_WARPS * 32);
    const T* rows = static_cast<const T*>(b->rows);
    for (const auto& c : b->i2_cls) {
        if (c.units == 0) continue;
        const dim3 grd(c.units);
        const void* fn = interp2_kernel<T, FORCE>(c.Pw, c.special);
        SE_CUDA(raise_smem_limit(fn, c.smem));
        const int P = c.special ? c.Pw : 0;
#define SE_I2ARGS b->sys, c.tab, b->srec, b->sg, b->perm, rows, b->boff, grid, \
                  out, phi, c.Ep, c.PL, c.zb
        if (P == 8) k_interp2<T, 8, FORCE><<<grd, blk, c.smem, st>>>(SE_I2ARGS);
        else if (P == 12) k_interp2<T, 12, FORCE><<<grd, blk, c.smem, st>>>(SE_I2ARGS);
        else if (P == 16) k_interp2<T, 16, FORCE><<<grd, blk, c.smem, st>>>(SE_I2ARGS);
        else k_interp2<T, 0, FORCE><<<grd, blk, c.smem, st>>>(SE_I2ARGS);
#undef SE_I2ARGS
        SE_CUDA(cudaGetLastError());
        LAUNCHED(b);
    }
    return SE_OK;
}

template <typename T>
static int launch_interp2(se_batch b, const T* grid, double* out, double* phi, cudaStream_t st)
{
    return b->i2_force ? launch_interp2_mode<T, true>(b, grid, out, phi, st)
                     : launch_interp2_mode<T, false>(b, grid, out, phi, st);
}

// grid32_fresh: grid32 holds the FP32 copy of `grid` already.
// grid32_ready: the FP32-FFT k-space step left the grids in grid32 (the FP64
// `grid` is then rebuilt from it only for the general interpolation).
static int run_interp(se_batch b, double* grid, double* out, double* phi, cudaStream_t st,
                      bool grid32_ready = false, bool grid32_fresh = false)
{
    if (b->ntot == 0) return SE_OK;
    // systems of whole 16^3 tiles with P <= 16: k_interp2 (FP32 path from an
    // FP32 copy of the grids); the others: k_interp / k_interp_global
    if (b->any_interp2) {
        if (b->precision == SE_FP32) {
            if (!grid32_ready && !grid32_fresh) SE_TRY(grid_f64_to_f32(b, grid, st));
            SE_TRY(launch_interp2<float>(b, b->grid32, out, phi, st));
        } else {
            SE_TRY(launch_interp2<double>(b, grid, out, phi, st));
        }
    }
    if (!b->any_interp1) return SE_OK;
    if (grid32_ready) SE_TRY(grid_f32_to_f64(b, grid, st));
    if (b->staged_interp) {
        if (b->precision == SE_FP32) return launch_interp_staged<float>(b, grid, out, phi, st);
        return launch_interp_staged<double>(b, grid, out, phi, st);
    }
    const unsigned nb = ceil_div(b->ntot, INTERP_WARPS);
    if (b->precision == SE_FP32)
        k_interp_global<float><<<nb, INTERP_WARPS * 32, 0, st>>>(
            b->sys, b->d_part_prefix, b->nsys, b->ntot, b->srec, b->sg, b->perm,
            static_cast<const float*>(b->fac), b->PS, static_cast<const float*>(b->rows), grid,
            out, phi);
    else
        k_interp_global<double><<<nb, INTERP_WARPS * 32, 0, st>>>(
            b->sys, b->d_part_prefix, b->nsys, b->ntot, b->srec, b->sg, b->perm,
            static_cast<const double*>(b->fac), b->PS, static_cast<const double*>(b->rows), grid,
            out, phi);
    SE_CUDA(cudaGetLastError());
    LAUNCHED(b);
    return SE_OK;
}

static int batch_solve_direct(se_batch b, const double* x, const double* q, double* out,
                              double* phi, cudaStream_t st)
{
    b->launches = b->pending_launches;
    b->pending_launches = 0;
    // stage events; inside a capture they become the graph's event-record
    // nodes (external records), so replays time the stages too
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (b->timing) SE_CUDA(cudaStreamIsCapturing(st, &cs));
    const unsigned rec_flags =
        cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
    auto mark = [&](int i) -> int {
        if (b->timing) SE_CUDA(cudaEventRecordWithFlags(b->ev[i], st, rec_flags));
        return SE_OK;
    };
    SE_CUDA(cudaMemsetAsync(b->err, 0, sizeof(int), st));
    SE_TRY(mark(0));
    SE_TRY(run_prepare_sort(b, x, q, st));
    SE_TRY(mark(1));
    SE_TRY(run_spread(b, b->grid, st));
    SE_TRY(mark(2));
    bool grid32_fresh = false;
    SE_TRY(run_kspace(b, b->grid, st, &grid32_fresh));
    SE_TRY(mark(3));
    SE_TRY(run_interp(b, b->grid, out, phi, st, b->fft32, grid32_fresh));
    SE_TRY(mark(4));
    return SE_OK;
}

// A solve through a CUDA graph: the launch sequence of a solve depends only
// on the buffers, the stream and the particle count (the systems' parameters
// are read from the device table), so a graph captured once replays every
// later solve with the same ones.  Slot 0 (the device-pointer entry points)
// replays only when graphs are on; the legacy default streams cannot be
// captured, and solves there run directly.
static int batch_solve(se_batch b, const double* x, const double* q, double* out, double* phi,
                       cudaStream_t st, int slot = 0)
{
    const bool capturable = st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread;
    if ((slot == 0 && !b->graph_on) || !capturable) return batch_solve_direct(b, x, q, out, phi, st);
    GraphSlot& g = b->gslot[slot];
    const bool same = g.stream == st && g.key[0] == x && g.key[1] == q && g.key[2] == out &&
                      g.key[3] == phi && g.ntot == b->ntot && g.timing == b->timing;
    if (!same) {
        graph_drop(g);
        g.stream = st;
        g.key[0] = x;
        g.key[1] = q;
        g.key[2] = out;
        g.key[3] = phi;
        g.ntot = b->ntot;
        g.timing = b->timing;
    }
    if (!g.exec && !g.warm) {   // first solve: direct (sets up kernel attributes)
        g.warm = true;
        return batch_solve_direct(b, x, q, out, phi, st);
    }
    const int pending = b->pending_launches;
    b->pending_launches = 0;
    if (!g.exec) {
        SE_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int r = batch_solve_direct(b, x, q, out, phi, st);
        cudaGraph_t gr = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &gr);
        if (r != SE_OK) {
            if (gr) cudaGraphDestroy(gr);
            return r;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        const cudaError_t ei = cudaGraphInstantiate(&g.exec, gr, 0);
        cudaGraphDestroy(gr);
        if (ei != cudaSuccess) {
            g.exec = nullptr;
            return cuda_fail(ei, "cudaGraphInstantiate", __FILE__, __LINE__);
        }
        g.launches = b->launches;
    }
    SE_CUDA(cudaGraphLaunch(g.exec, st));
    b->launches = pending + g.launches;
    return SE_OK;
}

static int set_graph(se_batch b, int on)
{
    if (!on) graph_drop(b->gslot[0]);
    b->graph_on = on != 0;
    return SE_OK;
}

static int set_timing(se_batch b, int on)
{
    if (on && !b->ev[0])
        for (auto& e : b->ev) SE_CUDA(cudaEventCreate(&e));
    b->timing = on != 0;
    return SE_OK;
}

static int stage_ms(se_batch b, float* ms)
{
    if (!b->timing || !ms) return SE_ERR_INVALID;
    SE_CUDA(cudaEventSynchronize(b->ev[4]));
    for (int i = 0; i < 4; i++) SE_CUDA(cudaEventElapsedTime(ms + i, b->ev[i], b->ev[i + 1]));
    return SE_OK;
}

// FP32 FMA throughput of this GPU: independent FMA chains in every thread of
// a grid that fills all SMs; the result is stored so nothing is elided.
__global__ void __launch_bounds__(256) k_fma_probe(float* out, int iters, float seed)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + threadIdx.x * 1e-7f + k;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], m, c);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace se

// ============================================================ C ABI =====

struct se_plan_s {
    se_config cfg;
    se_batch b = nullptr;
    // se_solve_host: device copies of the host buffers, the pinned input-error
    // flag, and the stream (with its fence event) its graph is captured on
    double* d_x = nullptr;
    double* d_q = nullptr;
    double* d_out = nullptr;
    int* h_err = nullptr;
    cudaStream_t hs = nullptr;
    cudaEvent_t hev = nullptr;
};

using namespace se;

// The error estimate SE_init_params prints (SE_general.c:517-572), Lindbo &
// Tornberg, for P points and c = m / sqrt(pi P) = 0.95.
static double se_error_bound(int P, double L, double xi, double Q, int mode)
{
    const double c = 0.95;
    const double g = exp(-PI_D * P * c * c / 2.);
    if (mode == SE_FORCE) return Q * sqrt(xi * L) / (L * L) * g * 2. * PI_D * c * c * P;
    return sqrt(Q * xi * L) / L * g;
}

extern "C" int se_choose_params(double eps, double L, double xi, double Q, int mode, int* M,
                                int* P, double* m)
{
    if (!(eps > 0) || !(L > 0) || !(xi > 0) || !(Q >= 0) || !M || !P || !m ||
        (mode != SE_POTENTIAL && mode != SE_FORCE))
        return SE_ERR_INVALID;
    int p = 2;
    while (p < MAX_P && se_error_bound(p, L, xi, Q, mode) > eps) p++;
    if (se_error_bound(p, L, xi, Q, mode) > eps) return SE_ERR_UNSUPPORTED;
    // Kolafa & Perram: the grid resolves the k-space sum to k_inf = 2 xi L
    int mm = (int)ceil(2. * (2. * xi * L) + 1.) + 2;
    mm = std::max(mm, p);
    mm = mm >= 32 ? (mm + 15) / 16 * 16 : (mm + 1) / 2 * 2;
    if (mm > 1024) return SE_ERR_UNSUPPORTED;
    *P = p;
    *M = mm;
    *m = 0.95 * sqrt(PI_D * p);
    return SE_OK;
}

extern "C" double se_error_estimate(int P, double L, double xi, double Q, int mode)
{
    return se_error_bound(P, L, xi, Q, mode);
}

extern "C" int se_config_derive(const se_config* cfg, double* h, double* w, double* eta,
                                double* c, double* d)
{
    if (!cfg || cfg->M < 1 || cfg->P < 1 || cfg->L <= 0 || cfg->m <= 0) return SE_ERR_INVALID;
    derive(cfg->M, cfg->P, cfg->L, cfg->xi, cfg->m, h, w, eta, c, d);
    return SE_OK;
}

static se_system sys_of(const se_config* c, int N)
{
    se_system s;
    s.N = N;
    s.M = c->M;
    s.P = c->P;
    s.L = c->L;
    s.xi = c->xi;
    s.m = c->m;
    s.mode = c->mode;
    return s;
}

extern "C" size_t se_plan_device_bytes(const se_config* cfg)
{
    if (!cfg) return 0;
    se_system s = sys_of(cfg, cfg->max_particles);
    return batch_bytes(&s, 1, cfg->precision, nullptr, nullptr) +
           (size_t)cfg->max_particles * 8 * 7;
}

extern "C" int se_plan_create(se_plan* plan, const se_config* cfg)
{
    if (!plan || !cfg || cfg->max_particles < 0) return SE_ERR_INVALID;
    se_system s = sys_of(cfg, cfg->max_particles);
    if (!valid_system(s)) return SE_ERR_INVALID;
    se_plan p = new se_plan_s();
    p->cfg = *cfg;
    int r = batch_create(&p->b, &s, 1, cfg->precision);
    if (r != SE_OK) {
        delete p;
        return r;
    }
    *plan = p;
    return SE_OK;
}

// ---------------------------------------------------------------- tuning --
// The kernel path of a plan chosen by timing: every valid path runs on the
// plan's configuration with synthetic uniform particles (N = its capacity, at
// most 2^20), and the fastest is kept in a process-wide table keyed by
// (M, P, mode, precision, ceil(log2 N)); with SE_GPU_TUNE_FILE set, the table
// is read from and appended to that file.

__global__ void k_tune_fill(double* __restrict__ x, double* __restrict__ q, int N, double L)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    for (int a = 0; a < 3; a++) {
        unsigned long long z = 0x9E3779B97F4A7C15ull * (3ull * n + a + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        x[n + (long long)a * N] = L * (double)(z >> 11) * (1.0 / 9007199254740992.0);
    }
    q[n] = (n & 1) ? -1.0 : 1.0;
}

namespace {

struct TuneKey {
    int M, P, mode, precision, nclass;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(M, P, mode, precision, nclass) <
               std::tie(o.M, o.P, o.mode, o.precision, o.nclass);
    }
};

std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;
bool g_tune_loaded = false;

const char* tune_file() { return getenv("SE_GPU_TUNE_FILE"); }

void tune_load()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* f = tune_file();
    if (!f) return;
    FILE* fp = fopen(f, "r");
    if (!fp) return;
    TuneKey k;
    int path;
    while (fscanf(fp, "%d %d %d %d %d %d", &k.M, &k.P, &k.mode, &k.precision, &k.nclass,
                  &path) == 6)
        if (path >= 0 && path <= 7) g_tune[k] = path;
    fclose(fp);
}

void tune_store(const TuneKey& k, int path)
{
    const char* f = tune_file();
    if (!f) return;
    FILE* fp = fopen(f, "a");
    if (!fp) return;
    fprintf(fp, "%d %d %d %d %d %d\n", k.M, k.P, k.mode, k.precision, k.nclass, path);
    fclose(fp);
}

int tune_candidates(int M, int P, int* c)
{
    if (!spread2_eligible(M, P)) {
        c[0] = 0;
        c[1] = PATH_RUNTIME_P;
        return 2;
    }
    const int all[6] = {PATH_TILE_SPREAD | PATH_PAIR_INTERP,
                        PATH_TILE_SPREAD | PATH_PAIR_INTERP | PATH_RUNTIME_P,
                        PATH_TILE_SPREAD, PATH_PAIR_INTERP, 0, PATH_RUNTIME_P};
    for (int i = 0; i < 6; i++) c[i] = all[i];
    return 6;
}

// Milliseconds of the fastest of 5 solves (after 2 untimed) on path `path`.
int time_path(const se_system& s, int precision, int path, const double* x, const double* q,
              double* out, cudaEvent_t e0, cudaEvent_t e1, float* best)
{
    se_batch b = nullptr;
    SE_TRY(batch_create(&b, &s, 1, precision, &path));
    int r = SE_OK;
    *best = 1e30f;
    for (int k = 0; k < 7 && r == SE_OK; k++) {
        cudaEventRecord(e0, nullptr);
        r = batch_solve_direct(b, x, q, out, nullptr, nullptr);
        cudaEventRecord(e1, nullptr);
        const cudaError_t e = cudaEventSynchronize(e1);
        if (r == SE_OK && e != cudaSuccess) r = cuda_fail(e, "tuning solve", __FILE__, __LINE__);
        float ms = 0;
        if (r == SE_OK && k >= 2 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
            *best = std::min(*best, ms);
    }
    batch_free(b);
    return r;
}

int tune_path(const se_config* cfg, int* path_out)
{
    std::lock_guard<std::mutex> g(g_tune_mu);
    tune_load();
    const int N = std::max(1, std::min(cfg->max_particles, 1 << 20));
    int nclass = 0;
    while ((1 << nclass) < std::max(cfg->max_particles, 1)) nclass++;
    const TuneKey key{cfg->M, cfg->P, cfg->mode, cfg->precision, nclass};
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
        *path_out = it->second;
        return SE_OK;
    }
    int cand[6];
    const int nc = tune_candidates(cfg->M, cfg->P, cand);
    se_system s = sys_of(cfg, N);
    double *x = nullptr, *q = nullptr, *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&x, sizeof(double) * 3 * N);
    if (e == cudaSuccess) e = cudaMalloc(&q, sizeof(double) * N);
    if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(double) * 3 * N);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    int r = e == cudaSuccess ? SE_OK : cuda_fail(e, "tuning buffers", __FILE__, __LINE__);
    if (r == SE_OK) {
        k_tune_fill<<<ceil_div(N, 256), 256>>>(x, q, N, cfg->L);
        e = cudaGetLastError();
        if (e != cudaSuccess) r = cuda_fail(e, "k_tune_fill", __FILE__, __LINE__);
    }
    int best_path = cand[0];
    float best_ms = 1e30f;
    for (int i = 0; i < nc && r == SE_OK; i++) {
        float ms = 0;
        r = time_path(s, cfg->precision, cand[i], x, q, out, e0, e1, &ms);
        if (r == SE_OK && ms < best_ms) {
            best_ms = ms;
            best_path = cand[i];
        }
    }
    if (x) cudaFree(x);
    if (q) cudaFree(q);
    if (out) cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (r != SE_OK) return r;
    g_tune[key] = best_path;
    tune_store(key, best_path);
    *path_out = best_path;
    return SE_OK;
}

}  // namespace

extern "C" int se_plan_create_ex(se_plan* plan, const se_config* cfg, int path)
{
    if (!plan || !cfg || cfg->max_particles < 0) return SE_ERR_INVALID;
    if (path == SE_PATH_DEFAULT) return se_plan_create(plan, cfg);
    se_system s = sys_of(cfg, cfg->max_particles);
    if (!valid_system(s) || (cfg->precision != SE_FP32 && cfg->precision != SE_FP64 &&
                             cfg->precision != SE_FP32_FFT32))
        return SE_ERR_INVALID;
    if (path == SE_PATH_TUNE) SE_TRY(tune_path(cfg, &path));
    if (path < 0 || path > 63) return SE_ERR_INVALID;
    se_plan p = new se_plan_s();
    p->cfg = *cfg;
    const int r = batch_create(&p->b, &s, 1, cfg->precision, &path);
    if (r != SE_OK) {
        delete p;
        return r;
    }
    *plan = p;
    return SE_OK;
}

extern "C" int se_plan_path(se_plan p) { return p ? p->b->host_sys[0].path : -1; }

extern "C" int se_plan_destroy(se_plan p)
{
    if (!p) return SE_OK;
    batch_free(p->b);
    if (p->hs) cudaStreamDestroy(p->hs);
    if (p->hev) cudaEventDestroy(p->hev);
    if (p->d_x) cudaFree(p->d_x);
    if (p->d_q) cudaFree(p->d_q);
    if (p->d_out) cudaFree(p->d_out);
    if (p->h_err) cudaFreeHost(p->h_err);
    delete p;
    return SE_OK;
}

// Stream-ordered rewrite of a single-system plan's device table: the
// kernels that follow on the stream see the new system, earlier ones the old.
__global__ void k_rebind(SysDev* sys, int* part_prefix, SysDev s)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *sys = s;
        part_prefix[1] = s.N;
    }
}

// Point a single-system plan at system s (same M, P and mode, N within the
// plan's capacity; L, xi, m and N free).  Nothing is issued when s is the
// system the plan already holds.
static int plan_rebind(se_plan p, const se_system& s, cudaStream_t st)
{
    if (!valid_system(s) || s.N > p->cfg.max_particles || s.M != p->cfg.M || s.P != p->cfg.P ||
        s.mode != p->cfg.mode)
        return SE_ERR_INVALID;
    se_batch b = p->b;
    SysDev S = b->host_sys[0];
    fill_sysdev(s, S);
    S.path = b->host_sys[0].path;   // the plan's kernel path stays
    if (memcmp(&S, &b->host_sys[0], sizeof(S)) == 0) return SE_OK;
    k_rebind<<<1, 32, 0, st>>>(b->sys, b->d_part_prefix, S);
    SE_CUDA(cudaGetLastError());
    b->pending_launches++;
    b->host_sys[0] = S;
    b->part_prefix[1] = s.N;
    b->ntot = s.N;
    return SE_OK;
}

static int plan_set_N(se_plan p, int N, cudaStream_t st)
{
    if (N < 0 || N > p->cfg.max_particles) return SE_ERR_INVALID;
    return plan_rebind(p, sys_of(&p->cfg, N), st);
}

extern "C" int se_solve(se_plan p, int N, const double* x, const double* q, double* out,
                        double* phi_out, void* stream)
{
    if (!p || (N > 0 && (!x || !q || !out))) return SE_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    SE_TRY(plan_set_N(p, N, st));
    return batch_solve(p->b, x, q, out, phi_out, st);
}

const int* se::plan_error_flag(se_plan p) { return p ? p->b->err : nullptr; }

extern "C" int se_solve_system(se_plan p, const se_system* sys, const double* x,
                               const double* q, double* out, double* phi_out, void* stream)
{
    if (!p || !sys || (sys->N > 0 && (!x || !q || !out))) return SE_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    SE_TRY(plan_rebind(p, *sys, st));
    return batch_solve(p->b, x, q, out, phi_out, st);
}

extern "C" int se_solve_host(se_plan p, int N, const double* xh, const double* qh,
                             double* outh, void* stream)
{
    if (!p || (N > 0 && (!xh || !qh || !outh))) return SE_ERR_INVALID;
    cudaStream_t user = as_stream(stream);
    const int cap = p->cfg.max_particles;
    const int outw = p->cfg.mode == SE_FORCE ? 3 : 1;
    if (!p->d_x) {
        SE_CUDA(cudaMalloc(&p->d_x, sizeof(double) * 3 * std::max(cap, 1)));
        SE_CUDA(cudaMalloc(&p->d_q, sizeof(double) * std::max(cap, 1)));
        SE_CUDA(cudaMalloc(&p->d_out, sizeof(double) * outw * std::max(cap, 1)));
        SE_CUDA(cudaMallocHost(&p->h_err, sizeof(int)));
        SE_CUDA(cudaStreamCreateWithFlags(&p->hs, cudaStreamNonBlocking));
        SE_CUDA(cudaEventCreateWithFlags(&p->hev, cudaEventDisableTiming));
    }
    // The call runs on the plan's own stream, after the work queued on the
    // caller's stream so far, and returns when it is done: the solve between
    // the copies replays the plan's host-entry graph (same device buffers and
    // stream every call; captured anew when N changes).  Pinned arrays are
    // copied by the stream itself; pageable ones through the pinned chunks
    // of host_to_device / device_to_host (threaded host copies), which
    // finish before the solve is queued and after it has finished.
    cudaStream_t st = p->hs;
    const bool pin_in = host_pinned(xh) && host_pinned(qh), pin_out = host_pinned(outh);
    SE_CUDA(cudaEventRecord(p->hev, user));
    SE_CUDA(cudaStreamWaitEvent(st, p->hev, 0));
    if (pin_in) {
        SE_CUDA(cudaMemcpyAsync(p->d_x, xh, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
        SE_CUDA(cudaMemcpyAsync(p->d_q, qh, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    } else {
        SE_CUDA(cudaStreamSynchronize(st));   // the caller's work first, as on the stream
        SE_TRY(host_to_device(p->d_x, xh, sizeof(double) * 3 * N));
        SE_TRY(host_to_device(p->d_q, qh, sizeof(double) * N));
    }
    SE_TRY(plan_set_N(p, N, st));
    SE_TRY(batch_solve(p->b, p->d_x, p->d_q, p->d_out, nullptr, st, 1));
    if (pin_out)
        SE_CUDA(cudaMemcpyAsync(outh, p->d_out, sizeof(double) * outw * N,
                                cudaMemcpyDeviceToHost, st));
    SE_CUDA(cudaMemcpyAsync(p->h_err, p->b->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SE_CUDA(cudaStreamSynchronize(st));
    if (!pin_out) SE_TRY(device_to_host(outh, p->d_out, sizeof(double) * outw * N));
    return *p->h_err ? SE_ERR_INPUT : SE_OK;
}

extern "C" int se_spread(se_plan p, int N, const double* x, const double* q, double* grid,
                         void* stream)
{
    if (!p || !grid || (N > 0 && (!x || !q))) return SE_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    SE_TRY(plan_set_N(p, N, st));
    p->b->launches = p->b->pending_launches;
    p->b->pending_launches = 0;
    SE_TRY(run_prepare_sort(p->b, x, q, st));
    // the tile kernels store 16-byte pairs: a caller grid that is not
    // 16-byte aligned is filled through the plan's own grid
    if (reinterpret_cast<uintptr_t>(grid) % 16 == 0) return run_spread(p->b, grid, st);
    SE_TRY(run_spread(p->b, p->b->grid, st));
    const long long M = p->cfg.M;
    SE_CUDA(cudaMemcpyAsync(grid, p->b->grid, sizeof(double) * M * M * M,
                            cudaMemcpyDeviceToDevice, st));
    return SE_OK;
}

extern "C" int se_kspace(se_plan p, double* grid, void* stream)
{
    if (!p || !grid) return SE_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    SE_TRY(run_kspace(p->b, grid, st));
    if (p->b->fft32) SE_TRY(grid_f32_to_f64(p->b, grid, st));   // the caller's grid is FP64
    return SE_OK;
}

extern "C" int se_interp(se_plan p, int N, const double* x, const double* q, const double* grid,
                         double* out, double* phi_out, void* stream)
{
    if (!p || !grid || (N > 0 && (!x || !q || !out))) return SE_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    SE_TRY(plan_set_N(p, N, st));
    p->b->launches = p->b->pending_launches;
    p->b->pending_launches = 0;
    SE_TRY(run_prepare_sort(p->b, x, q, st));
    // the window kernels read 16-byte groups: a caller grid that is not
    // 16-byte aligned is read through the plan's own grid
    if (reinterpret_cast<uintptr_t>(grid) % 16 != 0) {
        const long long M = p->cfg.M;
        SE_CUDA(cudaMemcpyAsync(p->b->grid, grid, sizeof(double) * M * M * M,
                                cudaMemcpyDeviceToDevice, st));
        grid = p->b->grid;
    }
    // only read: run_interp writes its grid argument when the FP32-FFT step left
    // the result in grid32, which is not the case here
    return run_interp(p->b, const_cast<double*>(grid), out, phi_out, st);
}

extern "C" int se_energy(const double* phi, const double* q, int N, double* e, void* stream)
{
    if (!phi || !q || !e || N < 0) return SE_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    static double* partial = nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!partial) SE_CUDA(cudaMalloc(&partial, sizeof(double) * 256));
    const int nb = std::min(256, std::max(1, (int)ceil_div(N, 256)));
    k_energy_partial<<<nb, 256, 0, st>>>(phi, q, N, partial);
    SE_CUDA(cudaGetLastError());
    k_energy_final<<<1, 256, 0, st>>>(partial, nb, e);
    SE_CUDA(cudaGetLastError());
    return SE_OK;
}

extern "C" int se_plan_launch_count(se_plan p) { return p ? p->b->launches : 0; }

extern "C" size_t se_batch_device_bytes(const se_system* systems, int nsys, int precision)
{
    if (!systems || nsys < 1) return 0;
    return batch_bytes(systems, nsys, precision, nullptr, nullptr);
}

extern "C" int se_batch_create(se_batch* b, const se_system* systems, int nsys, int precision)
{
    return batch_create(b, systems, nsys, precision);
}

extern "C" int se_default_path(int M, int P) { return default_path(M, P); }

extern "C" int se_batch_create_ex(se_batch* b, const se_system* systems, int nsys,
                                  int precision, const int* paths)
{
    return batch_create(b, systems, nsys, precision, paths);
}

extern "C" int se_batch_destroy(se_batch b) { return batch_free(b); }

extern "C" int se_batch_solve(se_batch b, const double* x, const double* q, double* out,
                              void* stream)
{
    if (!b || (b->ntot > 0 && (!x || !q || !out))) return SE_ERR_INVALID;
    return batch_solve(b, x, q, out, nullptr, as_stream(stream));
}

extern "C" int se_batch_launch_count(se_batch b) { return b ? b->launches : 0; }

extern "C" int se_plan_set_graph(se_plan p, int on)
{
    return p ? set_graph(p->b, on) : SE_ERR_INVALID;
}

extern "C" int se_batch_set_graph(se_batch b, int on)
{
    return b ? set_graph(b, on) : SE_ERR_INVALID;
}

extern "C" int se_plan_set_timing(se_plan p, int on)
{
    return p ? set_timing(p->b, on) : SE_ERR_INVALID;
}

extern "C" int se_plan_stage_ms(se_plan p, float* ms)
{
    return p ? stage_ms(p->b, ms) : SE_ERR_INVALID;
}

extern "C" int se_batch_set_timing(se_batch b, int on)
{
    return b ? set_timing(b, on) : SE_ERR_INVALID;
}

extern "C" int se_batch_stage_ms(se_batch b, float* ms) { return b ? stage_ms(b, ms) : SE_ERR_INVALID; }

extern "C" int se_probe_fma_tflops(double* tflops, void* stream)
{
    if (!tflops) return SE_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    int dev = 0, sms = 0;
    SE_CUDA(cudaGetDevice(&dev));
    SE_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    float* out = nullptr;
    SE_CUDA(cudaMalloc(&out, sizeof(float) * blocks * threads));
    cudaEvent_t e0, e1;
    SE_CUDA(cudaEventCreate(&e0));
    SE_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        SE_CUDA(cudaEventRecord(e0, st));
        k_fma_probe<<<blocks, threads, 0, st>>>(out, iters, 1.0f + r);
        SE_CUDA(cudaGetLastError());
        SE_CUDA(cudaEventRecord(e1, st));
        SE_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        SE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (r > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return SE_OK;
}

extern "C" const char* se_gpu_error_detail(void) { return se::g_err_msg; }
