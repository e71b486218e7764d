// se_device.cuh -- definitions shared by the device-resident kernels
// (included inside namespace se by se_solve.cu).
#pragma once

constexpr int FB = 8;                     // fine bin edge, in stencil corners
constexpr int TX = 16, TY = 16, TZ = 16;  // spread tile (output cells)
constexpr int WY = 4, WZ = 8;             // one warp's lane block: 4 y x 8 z
constexpr int SPREAD_WARPS = (TY / WY) * (TZ / WZ);
constexpr int SPREAD_THREADS = SPREAD_WARPS * 32;
// particles staged per spread round
template <typename Acc>
constexpr int spread_chunk() { return 64; }

// Packed FP32 pairs (sm_100a): one FFMA2 (__ffma2_rn) does two FP32 FMAs,
// each rounded to nearest.
__device__ __forceinline__ float2 f32x2(float lo, float hi) { return make_float2(lo, hi); }

__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// The two packed pairs in 16 bytes of FP32 values.
__device__ __forceinline__ void f32x2_split(const float4& v, float2& lo, float2& hi)
{
    lo = make_float2(v.x, v.y);
    hi = make_float2(v.z, v.w);
}

// The tile-aligned kernels (k_spread2, k_interp2 on tile-aligned factor rows)
// apply when a system's grid is cut into whole 16^3 tiles and its stencil
// fits two tiles.
__host__ __device__ inline bool spread2_eligible(int M, int P)
{
    return M % 16 == 0 && M >= 32 && P <= 16;
}

// A system's kernel path (SysDev::path): which spread and interpolation run.
constexpr int PATH_TILE_SPREAD = 1;    // k_spread2 (else k_spread)
constexpr int PATH_PAIR_INTERP = 2;    // k_interp2 (else k_interp / k_interp_global)
constexpr int PATH_RUNTIME_P = 4;      // interpolation without the P-unrolled variants
constexpr int PATH_RADIX_SORT = 8;     // the batch sorts with the radix passes (se_sort.cu)
constexpr int PATH_FFT3 = 16;          // the batch's FP64 FFTs through se_fft.cuh (not cuFFT)
constexpr int PATH_BIN_WINDOWS = 32;   // k_interp2 stages one window per bin (not per z pair)

// The default path: the tile-aligned spread wherever it applies, and the
// window-pair interpolation from P = 8 on (for shorter stencils its
// per-particle set-up and z-pair padding cost more than they save: the timed
// choice picks the general interpolation there on B200).
__host__ __device__ inline int default_path(int M, int P)
{
    if (!spread2_eligible(M, P)) return 0;
    return PATH_TILE_SPREAD | (P >= 8 ? PATH_PAIR_INTERP : 0);
}

constexpr int MAX_SEG = 96;               // bin segments reaching one tile
constexpr int INTERP_WARPS = 8;
constexpr int MAX_P = 32;
constexpr double PI_D = 3.14159265358979323846;

// Per-system parameters and offsets of a batch (one entry per system).
struct SysDev {
    int N, M, P, lo, mode;
    int path;         // PATH_* bits
    int part_off, out_off;
    long long grid_off, spec_off;
    int nf[3];        // fine bins per axis
    int bin_base;     // first global fine-bin id
    int nt[3];        // spread tiles per axis
    int tile_base;    // first global spread-tile id
    double h, c, d, h3;
    double rho;       // exp(-2 c h^2)
    double kfac;      // 2 pi / L
    double scalar;    // -(1 - eta) / (4 xi^2)
    double dnorm;     // 4 pi / M^3
};

// largest s with prefix[s] <= v
__device__ __forceinline__ int find_sys(const int* __restrict__ prefix, int nsys, int v)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// periodic index in [0, n) for any int i (SE_fgg.c:17-25 vmod)
__device__ __forceinline__ int pmod(int i, int n)
{
    const int r = i % n;
    return r < 0 ? r + n : r;
}

// i in (-n, 2n) to [0, n) without a division
__device__ __forceinline__ int wrap1(int i, int n)
{
    i = i < 0 ? i + n : i;
    return i >= n ? i - n : i;
}

__device__ __forceinline__ int pack_g(int gx, int gy, int gz) { return gx | (gy << 10) | (gz << 20); }
__device__ __forceinline__ int g_of(int pk, int a) { return (pk >> (10 * a)) & 1023; }
