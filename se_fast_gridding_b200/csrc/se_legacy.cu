// se_legacy.cu -- the SE_fast_gridding C API (SE_fgg.h, SE_general.h) on B200.
//
// Each exported symbol keeps the reference's name, arguments and meaning (the
// declaration in include/se_fgg_gpu.h cites the function it replaces).  The
// arithmetic runs in FP64 CUDA kernels that keep the reference's operation
// order inside every product and sum where the order is fixed there (wrap,
// the expansion recurrences); scatter sums use FP64 atomics, so only the
// order of the additions into a grid cell can differ (rounding level).
//
// Pointers may be host, pinned, managed or device memory.  Host buffers are
// staged through pooled device mirrors inside each call (the copies
// pipelined through pinned chunks, se_hoststage.cu); managed and device
// buffers are used in place.  Every call ends with its outputs visible to the
// host (synchronous, as the reference is).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>
#include <sys/time.h>

#include "se_fgg_gpu.h"
#include "se_internal.h"

namespace se {
namespace legacy {

constexpr double PI_D = 3.14159265358979323846;

// ---------------------------------------------------------- last error ---

static thread_local int t_err = 0;
static thread_local char t_msg[256] = "";

static void set_error(int code, const char* msg)
{
    t_err = code;
    snprintf(t_msg, sizeof(t_msg), "%s", msg);
    if (code) fprintf(stderr, "[se_gpu] %s\n", msg);
}

// The periodicity of the names the reference builds per periodicity
// (SE_FGG_expand_all, SE_FGG_grid, SE_FGG_int: -DTHREE_PERIODIC,
// -DTWO_PERIODIC or -DONE_PERIODIC, SE_fgg.h:17-33): SE_GPU_PERIODICITY = 2 or
// 1 selects 2P or 1P, anything else 3P.
static int periodicity_default()
{
    static int p = [] {
        const char* e = getenv("SE_GPU_PERIODICITY");
        const int v = e ? atoi(e) : 3;
        return (v == 2 || v == 1) ? v : 3;
    }();
    return p;
}

// ------------------------------------------------------ pointer staging ---

static bool on_device(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device buffers that stand in for the caller's host arrays during a call.
// A call takes them from this pool and gives them back when it returns (its
// outputs are in host memory by then), so a caller that passes new host
// arrays on every call -- spectral_ewald() mallocs its grids per solve --
// reuses the same device memory instead of allocating it again.  Idle
// buffers beyond LIMIT bytes are freed, largest first.
struct MirrorPool {
    std::mutex mu;
    std::multimap<size_t, void*> idle;   // capacity -> buffer
    size_t idle_bytes = 0;
    static constexpr size_t LIMIT = size_t(16) << 30;

    int acquire(size_t bytes, void** d, size_t* cap)
    {
        {
            std::lock_guard<std::mutex> lock(mu);
            auto it = idle.lower_bound(bytes);
            if (it != idle.end() && it->first <= 2 * bytes) {   // best fit, at most 2x
                *d = it->second;
                *cap = it->first;
                idle_bytes -= it->first;
                idle.erase(it);
                return SE_OK;
            }
        }
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(mirror)", __FILE__, __LINE__);
        *d = p;
        *cap = bytes;
        return SE_OK;
    }

    void release(void* d, size_t cap)
    {
        std::lock_guard<std::mutex> lock(mu);
        idle.emplace(cap, d);
        idle_bytes += cap;
        while (idle_bytes > LIMIT && !idle.empty()) {
            auto it = std::prev(idle.end());
            cudaFree(it->second);
            idle_bytes -= it->first;
            idle.erase(it);
        }
    }
};

static MirrorPool& mirrors()
{
    static MirrorPool* c = new MirrorPool();
    return *c;
}

// Collects the buffers of one call, copies host inputs in, copies host
// outputs back at the end (se_hoststage.cu), and returns the device mirrors
// to the pool when it goes out of scope.  The same pointer used twice shares
// one mirror.
class Stager {
public:
    Stager() = default;
    Stager(const Stager&) = delete;
    Stager& operator=(const Stager&) = delete;
    ~Stager()
    {
        for (auto& e : ents_)
            if (e.host && e.d) mirrors().release(e.d, e.cap);
    }
    void* use(const void* h, size_t bytes, bool in, bool out)
    {
        if (!h || bytes == 0 || err_) return nullptr;
        for (auto& e : ents_)
            if (e.h == h) {
                if (bytes > e.bytes) {   // grow: take a larger mirror
                    e.bytes = bytes;
                    if (e.host && bytes > e.cap) {
                        mirrors().release(e.d, e.cap);
                        e.d = nullptr;
                        if ((err_ = mirrors().acquire(bytes, &e.d, &e.cap))) return nullptr;
                    }
                }
                e.in |= in;
                e.out |= out;
                return e.d;
            }
        Ent e{h, nullptr, bytes, 0, !on_device(h), in, out};
        if (e.host) {
            if ((err_ = mirrors().acquire(bytes, &e.d, &e.cap))) return nullptr;
        } else {
            e.d = const_cast<void*>(h);
        }
        ents_.push_back(e);
        return e.d;
    }
    int copy_in();
    int finish();
    int error() const { return err_; }

private:
    struct Ent {
        const void* h;
        void* d;
        size_t bytes, cap;   // cap: the mirror's size (host arrays)
        bool host, in, out;
    };
    std::vector<Ent> ents_;
    int err_ = 0;
};

static void report(int code, const char* fn)
{
    if (code == SE_OK) {
        t_err = 0;
        t_msg[0] = 0;
        return;
    }
    char buf[200];
    snprintf(buf, sizeof(buf), "%s failed (code %d)", fn, code);
    set_error(code, buf);
}

static bool valid_params(const SE_FGG_params* p)
{
    if (!p || p->P < 1 || p->P > SE_P_MAX || p->N < 0) return false;
    for (int d = 0; d < 3; d++)
        if (p->dims[d] < 1 || p->npdims[d] < 1) return false;
    return true;
}

static size_t npad(const SE_FGG_params* p)
{
    return (size_t)p->npdims[0] * p->npdims[1] * p->npdims[2];
}

static size_t nper(const SE_FGG_params* p)
{
    return (size_t)p->dims[0] * p->dims[1] * p->dims[2];
}

// Elements of the periodic grid a wrap writes / an extend reads: 3P
// M0 M1 M2; 2P M0 M1 (M2 + P); 1P the largest index of the reference's
// column-major map i + j M0 + k M0 M1 over the unfolded i < M0 + P,
// j < M1 + P (SE_fgg.c:387-411, :478-502 index H_per with the periodic
// strides M0, M1 over the padded x and y extents, so the map overlaps itself
// and runs P M0 + P - 1 past M0 M1 M2).
static long long nper_of(const SE_FGG_params* p, int periodicity)
{
    const long long m0 = p->dims[0], m1 = p->dims[1], m2 = p->dims[2];
    if (periodicity == 2) return m0 * m1 * p->npdims[2];
    if (periodicity == 1)
        return (p->npdims[0] - 1) + (p->npdims[1] - 1) * m0 + (m2 - 1) * m0 * m1 + 1;
    return m0 * m1 * m2;
}

// ------------------------------------------------------------- kernels ---

__device__ __forceinline__ int vmod_d(int i, int n)
{
    const int r = i % n;
    return r < 0 ? r + n : r;
}

struct ParamsDev {
    int N, P, P_half, lo;   // lo: first stencil offset (-p_half or 1 - p_half)
    int dims[3], npdims[3];
    double c, d, h, a, b;   // a, b: offsets of the free directions (2P: z; 1P: x, y)
};

// Set by a kernel that skipped a particle whose stencil leaves the padded
// grid (positions outside [0, L] give such indices; the reference writes out
// of bounds there).  Reset and read by every legacy call.
__device__ int g_legacy_err;

__device__ __forceinline__ bool stencil_in_bounds(long long base, const ParamsDev& p)
{
    const long long n = (long long)p.npdims[0] * p.npdims[1] * p.npdims[2];
    const long long last =
        base + ((long long)(p.P - 1) * p.npdims[1] + (p.P - 1)) * p.npdims[2] + (p.P - 1);
    return base >= 0 && last < n;
}

int Stager::copy_in()
{
    if (err_) return err_;
    const int zero = 0;
    SE_CUDA(cudaMemcpyToSymbol(g_legacy_err, &zero, sizeof(int)));
    for (auto& e : ents_)
        if (e.host && e.in) SE_TRY(host_to_device(e.d, e.h, e.bytes));
    return SE_OK;
}

int Stager::finish()
{
    if (err_) return err_;
    SE_CUDA(cudaGetLastError());
    SE_CUDA(cudaDeviceSynchronize());
    for (auto& e : ents_)
        if (e.host && e.out) SE_TRY(device_to_host(const_cast<void*>(e.h), e.d, e.bytes));
    int flag = 0;
    SE_CUDA(cudaMemcpyFromSymbol(&flag, g_legacy_err, sizeof(int)));
    return flag ? SE_ERR_INPUT : SE_OK;
}

static ParamsDev to_dev(const SE_FGG_params* p)
{
    ParamsDev q;
    q.N = p->N;
    q.P = p->P;
    q.P_half = p->P_half;
    const int ph = (p->P & 1) ? (p->P - 1) / 2 : p->P / 2;
    q.lo = (p->P & 1) ? -ph : -ph + 1;
    for (int d = 0; d < 3; d++) {
        q.dims[d] = p->dims[d];
        q.npdims[d] = p->npdims[d];
    }
    q.c = p->c;
    q.d = p->d;
    q.h = p->h;
    q.a = p->a;
    q.b = p->b;
    return q;
}

// SE_fgg.c:508-535
__global__ void k_base_gaussian(double* zs, ParamsDev p)
{
    const int P = p.P;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P * P * P) return;
    const int ph = (P & 1) ? (P - 1) / 2 : P / 2;
    const int from = (P & 1) ? ph : ph - 1;
    const int i = t / (P * P) - from, j = (t / P) % P - from, k = t % P - from;
    const double a = i * p.h, b = j * p.h, e = k * p.h;
    zs[t] = p.d * exp(-p.c * (a * a + b * b + e * e));
}

// One particle's expansion, SE_fgg.c:539-621 (3P), :625-722 (force),
// :727-819 (2P: z free, offset a), :823-916 (1P: x and y free, offsets a
// and b); q folded into zx.  Returns the padded corner index.
__device__ int expand_one(const double xn[3], double q, const ParamsDev& p, int periodicity,
                          double* zx, double* zy, double* zz, double* zfx, double* zfy,
                          double* zfz)
{
    const int P = p.P, ph = p.P_half;
    const bool odd = P & 1;
    double t0[3];
    int first[3];
    for (int d = 0; d < 3; d++) {
        const bool sh = (periodicity == 2 && d == 2) || (periodicity == 1 && d < 2);
        const double s = sh ? (periodicity == 1 && d == 1 ? p.b : p.a) + p.h / 2 : 0.0;
        const double u = sh ? (xn[d] - s) / p.h : xn[d] / p.h;
        const int cell = odd ? (int)round(u) : (int)floor(u);
        first[d] = odd ? cell - ph : cell - (ph - 1);
        t0[d] = sh ? xn[d] - (cell * p.h + s) : xn[d] - p.h * cell;
    }
    const double z3 = exp(-p.c * (t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2])) * q;
    double* z[3] = {zx, zy, zz};
    double* zf[3] = {zfx, zfy, zfz};
    for (int d = 0; d < 3; d++) {
        const double base = exp(2 * p.c * p.h * t0[d]);
        double v = pow(base, (double)p.lo);
        z[d][0] = v;
        for (int i = 1; i < P; i++) {
            v *= base;
            z[d][i] = v;
        }
        if (zf[d])
            for (int i = 0; i < P; i++) zf[d][i] = -p.c * (t0[d] - (p.lo + i) * p.h);
    }
    for (int i = 0; i < P; i++) zx[i] *= z3;
    if (periodicity == 1)   // the free x and y corners are not shifted (:912-915)
        return (first[0] * p.npdims[1] + first[1]) * p.npdims[2] + first[2] + ph;
    const int kz = periodicity == 2 ? first[2] : first[2] + ph;
    return ((first[0] + ph) * p.npdims[1] + first[1] + ph) * p.npdims[2] + kz;
}

// SE_fgg.c:920-963 (q = 1)
__global__ void k_expand_all(ParamsDev p, const double* __restrict__ x, int periodicity,
                             double* zx, double* zy, double* zz, double* zfx, double* zfy,
                             double* zfz, int* idx)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= p.N) return;
    const double xn[3] = {x[n], x[n + p.N], x[n + 2 * p.N]};
    const long long o = (long long)n * p.P;
    idx[n] = expand_one(xn, 1.0, p, periodicity, zx + o, zy + o, zz + o,
                        zfx ? zfx + o : nullptr, zfy ? zfy + o : nullptr,
                        zfz ? zfz + o : nullptr);
}

// Scatter of one particle's P^3 stencil per CTA.  force_order selects the
// product order of SE_fgg.c:4964-5009 instead of :3983-4028.
__global__ void k_grid_split(double* H, const double* __restrict__ q,
                             const double* __restrict__ zs, const double* __restrict__ zx,
                             const double* __restrict__ zy, const double* __restrict__ zz,
                             const int* __restrict__ idx, ParamsDev p, int force_order)
{
    const int n = blockIdx.x;
    const int P = p.P;
    const long long o = (long long)n * P;
    const double qn = q[n];
    const long long base = idx[n];
    if (!stencil_in_bounds(base, p)) {
        if (threadIdx.x == 0) atomicOr(&g_legacy_err, 1);
        return;
    }
    const int n1 = p.npdims[1], n2 = p.npdims[2];
    for (int s = threadIdx.x; s < P * P * P; s += blockDim.x) {
        const int i = s / (P * P), j = (s / P) % P, k = s % P;
        double v;
        if (force_order) {
            const double cij = zx[o + i] * zy[o + j];
            v = zs[s] * zz[o + k] * cij * qn;
        } else {
            const double cij = qn * zx[o + i] * zy[o + j];
            v = zs[s] * zz[o + k] * cij;
        }
        atomicAdd(H + base + ((long long)i * n1 + j) * n2 + k, v);
    }
}

// SE_fgg.c:3866-3914: expansion with the charge, then the same scatter
__global__ void k_grid_vanilla(double* H, const double* __restrict__ x,
                               const double* __restrict__ q, const double* __restrict__ zs,
                               ParamsDev p, int periodicity)
{
    __shared__ double z[3][SE_P_MAX];
    __shared__ int c0;
    const int n = blockIdx.x;
    const int P = p.P;
    if (threadIdx.x == 0) {
        const double xn[3] = {x[n], x[n + p.N], x[n + 2 * p.N]};
        c0 = expand_one(xn, q[n], p, periodicity, z[0], z[1], z[2], nullptr, nullptr, nullptr);
    }
    __syncthreads();
    if (!stencil_in_bounds(c0, p)) {
        if (threadIdx.x == 0) atomicOr(&g_legacy_err, 1);
        return;
    }
    const int n1 = p.npdims[1], n2 = p.npdims[2];
    for (int s = threadIdx.x; s < P * P * P; s += blockDim.x) {
        const int i = s / (P * P), j = (s / P) % P, k = s % P;
        const double cij = z[0][i] * z[1][j];
        atomicAdd(H + c0 + ((long long)i * n1 + j) * n2 + k, zs[s] * z[2][k] * cij);
    }
}

// SE_fgg.c:327-352 / :357-382 / :387-411 as a gather: each periodic cell adds
// its padded pre-images in the reference's row-major order.
__global__ void k_wrap(double* H_per, const double* __restrict__ H, ParamsDev p,
                       int periodicity, long long nout)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nout) return;
    const int m0 = p.dims[0], m1 = p.dims[1], m2 = p.dims[2];
    const int n0 = p.npdims[0], n1 = p.npdims[1], n2 = p.npdims[2];
    const int ph = (p.P & 1) ? (p.P - 1) / 2 : p.P / 2;
    if (periodicity == 1) {
        // pre-images (i, j, k) of c = i + m0 (j + m1 w), w = vmod(k - ph, m2),
        // i < n0, j < n1, k < n2, walked with i, then j, then k ascending
        double acc = H_per[c];
        for (long long i = c % m0; i < n0 && i <= c; i += m0) {
            const long long sv = (c - i) / m0;   // j + m1 w
            for (long long j = sv % m1; j < n1 && j <= sv; j += m1) {
                const long long w = (sv - j) / m1;
                if (w >= m2) continue;
                const long long row = (i * n1 + j) * n2;
                for (int k = vmod_d((int)w + ph, m2); k < n2; k += m2) acc += H[row + k];
            }
        }
        H_per[c] = acc;
        return;
    }
    const int wi = (int)(c % m0);
    const int wj = (int)((c / m0) % m1);
    const int wk = (int)(c / ((long long)m0 * m1));
    double acc = H_per[c];
    for (int i = vmod_d(wi + ph, m0); i < n0; i += m0)
        for (int j = vmod_d(wj + ph, m1); j < n1; j += m1) {
            const long long row = ((long long)i * n1 + j) * n2;
            if (periodicity == 2) {
                acc += H[row + wk];
            } else {
                for (int k = vmod_d(wk + ph, m2); k < n2; k += m2) acc += H[row + k];
            }
        }
    H_per[c] = acc;
}

// SE_fgg.c:417-443 / :448-473 / :478-502
__global__ void k_extend(double* H, const double* __restrict__ H_per, ParamsDev p,
                         int periodicity, int ph)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n0 = p.npdims[0], n1 = p.npdims[1], n2 = p.npdims[2];
    if (t >= (long long)n0 * n1 * n2) return;
    const int k = (int)(t % n2), j = (int)((t / n2) % n1), i = (int)(t / ((long long)n1 * n2));
    const int m0 = p.dims[0], m1 = p.dims[1], m2 = p.dims[2];
    if (periodicity == 1) {
        H[t] = H_per[i + (long long)m0 * (j + (long long)m1 * vmod_d(k - ph, m2))];
        return;
    }
    const int wi = vmod_d(i - ph, m0), wj = vmod_d(j - ph, m1);
    const int wk = periodicity == 2 ? k : vmod_d(k - ph, m2);
    H[t] = H_per[wi + (long long)m0 * (wj + (long long)m1 * wk)];
}

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// SE_fgg.c:1176-1223 (one warp per particle); accumulate: SE_fgg.c:1856
__global__ void k_int_split(double* phi, const double* __restrict__ H,
                            const double* __restrict__ zs, const double* __restrict__ zx,
                            const double* __restrict__ zy, const double* __restrict__ zz,
                            const int* __restrict__ idx, ParamsDev p, double h3, int accumulate)
{
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (m >= p.N) return;
    const int P = p.P, n1 = p.npdims[1], n2 = p.npdims[2];
    const long long o = (long long)m * P;
    const long long base = idx[m];
    if (!stencil_in_bounds(base, p)) {
        if (lane == 0) atomicOr(&g_legacy_err, 1);
        return;
    }
    double acc = 0;
    for (int s = lane; s < P * P * P; s += 32) {
        const int i = s / (P * P), j = (s / P) % P, k = s % P;
        const double cij = zx[o + i] * zy[o + j];
        acc += H[base + ((long long)i * n1 + j) * n2 + k] * zs[s] * zz[o + k] * cij;
    }
    acc = warp_sum_d(acc);
    if (lane == 0) phi[m] = accumulate ? phi[m] + h3 * acc : h3 * acc;
}

// SE_fgg.c:968-1019 (expansion recomputed, q = 1)
__global__ void k_int_vanilla(double* phi, const double* __restrict__ H,
                              const double* __restrict__ x, const double* __restrict__ zs,
                              ParamsDev p, int periodicity, double h3)
{
    __shared__ double z[8][3][SE_P_MAX];
    __shared__ int c0s[8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = blockIdx.x * 8 + w;
    if (m >= p.N) return;
    if (lane == 0) {
        const double xm[3] = {x[m], x[m + p.N], x[m + 2 * p.N]};
        c0s[w] = expand_one(xm, 1.0, p, periodicity, z[w][0], z[w][1], z[w][2], nullptr,
                            nullptr, nullptr);
    }
    __syncwarp();
    const int P = p.P, n1 = p.npdims[1], n2 = p.npdims[2];
    const long long base = c0s[w];
    if (!stencil_in_bounds(base, p)) {
        if (lane == 0) atomicOr(&g_legacy_err, 1);
        return;
    }
    double acc = 0;
    for (int s = lane; s < P * P * P; s += 32) {
        const int i = s / (P * P), j = (s / P) % P, k = s % P;
        const double cij = z[w][0][i] * z[w][1][j];
        acc += H[base + ((long long)i * n1 + j) * n2 + k] * zs[s] * z[w][2][k] * cij;
    }
    acc = warp_sum_d(acc);
    if (lane == 0) phi[m] = h3 * acc;
}

// SE_fgg.c:2241-2312
__global__ void k_int_split_force(double* force, const double* __restrict__ q,
                                  const double* __restrict__ H, const double* __restrict__ zs,
                                  const double* __restrict__ zx, const double* __restrict__ zy,
                                  const double* __restrict__ zz, const double* __restrict__ zfx,
                                  const double* __restrict__ zfy,
                                  const double* __restrict__ zfz, const int* __restrict__ idx,
                                  ParamsDev p, double h3)
{
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (m >= p.N) return;
    const int P = p.P, n1 = p.npdims[1], n2 = p.npdims[2];
    const long long o = (long long)m * P;
    const long long base = idx[m];
    if (!stencil_in_bounds(base, p)) {
        if (lane == 0) atomicOr(&g_legacy_err, 1);
        return;
    }
    const double qm = q[m];
    double f0 = 0, f1 = 0, f2 = 0;
    for (int s = lane; s < P * P * P; s += 32) {
        const int i = s / (P * P), j = (s / P) % P, k = s % P;
        const double cij = zx[o + i] * zy[o + j];
        const double t = H[base + ((long long)i * n1 + j) * n2 + k] * zs[s] * zz[o + k] * cij * qm;
        f0 += t * zfx[o + i];
        f1 += t * zfy[o + j];
        f2 += t * zfz[o + k];
    }
    f0 = warp_sum_d(f0);
    f1 = warp_sum_d(f1);
    f2 = warp_sum_d(f2);
    if (lane == 0) {
        force[m] = h3 * f0;
        force[m + p.N] = h3 * f1;
        force[m + 2 * p.N] = h3 * f2;
    }
}

// SE_fgg.c:1024-1100 (3P force expansion with the charge)
__global__ void k_int_force_vanilla(double* force, const double* __restrict__ H,
                                    const double* __restrict__ x, const double* __restrict__ q,
                                    const double* __restrict__ zs, ParamsDev p, double h3)
{
    __shared__ double z[4][6][SE_P_MAX];
    __shared__ int c0s[4];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = blockIdx.x * 4 + w;
    if (m >= p.N) return;
    if (lane == 0) {
        const double xm[3] = {x[m], x[m + p.N], x[m + 2 * p.N]};
        c0s[w] = expand_one(xm, q[m], p, 3, z[w][0], z[w][1], z[w][2], z[w][3], z[w][4],
                            z[w][5]);
    }
    __syncwarp();
    const int P = p.P, n1 = p.npdims[1], n2 = p.npdims[2];
    const long long base = c0s[w];
    if (!stencil_in_bounds(base, p)) {
        if (lane == 0) atomicOr(&g_legacy_err, 1);
        return;
    }
    double f0 = 0, f1 = 0, f2 = 0;
    for (int s = lane; s < P * P * P; s += 32) {
        const int i = s / (P * P), j = (s / P) % P, k = s % P;
        const double cij = z[w][0][i] * z[w][1][j];
        const double t = H[base + ((long long)i * n1 + j) * n2 + k] * zs[s] * z[w][2][k] * cij;
        f0 += t * z[w][3][i];
        f1 += t * z[w][4][j];
        f2 += t * z[w][5][k];
    }
    f0 = warp_sum_d(f0);
    f1 = warp_sum_d(f1);
    f2 = warp_sum_d(f2);
    if (lane == 0) {
        force[m] = h3 * f0;
        force[m + p.N] = h3 * f1;
        force[m + 2 * p.N] = h3 * f2;
    }
}

// SE_general.c:145-175, indices as there (Z[i*n3*n2 + j*n2 + k])
__global__ void k_scaling(double* Z, int n1, int n2, int n3, double f0, double f1, double f2,
                          double scalar)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)n1 * n2 * n3;
    if (t >= n) return;
    const int k = (int)(t % n3), j = (int)((t / n3) % n2), i = (int)(t / ((long long)n2 * n3));
    // k_vec(n1, ...) fills all three axes with n1 points
    const int npos = (n1 % 2 == 0) ? n1 / 2 : (n1 - 1) / 2 + 1;
    const double ki = f0 * (double)(i < npos ? i : i - n1);
    const double kj = f1 * (double)(j < npos ? j : j - n1);
    const double kk = f2 * (double)(k < npos ? k : k - n1);
    const double d = 4. * PI_D / (double)(n1 * n1 * n1);
    const double K2 = (ki * ki + kj * kj) + kk * kk;
    Z[(long long)i * n3 * n2 + (long long)j * n2 + k] = exp(scalar * K2) / K2 * d;
}

__global__ void k_product_rc(double2* c, const double2* a, const double* b, long long n, int flag)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double2 v = a[t];
    if (flag == -1) {
        v.x = v.x / b[t];
        v.y = v.y / b[t];
    } else {
        v.x = v.x * b[t];
        v.y = v.y * b[t];
    }
    c[t] = v;
}

__global__ void k_copy_r2c(const double* in, double2* out, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = make_double2(in[t], 0.0);
}

__global__ void k_copy_c2r(const double2* in, double* out, long long n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = in[t].x;
}

__global__ void k_permute_state(double* x, double* q, const double* xc, const double* qc,
                                const int* perm, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int j = perm[i];
    x[i] = xc[j];
    x[i + N] = xc[j + N];
    x[i + 2 * N] = xc[j + 2 * N];
    q[i] = qc[j];
}

__global__ void k_key_shift(const int* idx, int* keys, int N, int lo)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) keys[i] = idx[i] - lo;
}

// ------------------------------------------------------------ helpers ----

static unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// POTENTIAL int dispatch of the AVX build (SE_fgg.c:1710-1764): only the
// unroll-4 kernel (P % 4 == 0, not 8/16/unroll-8) accumulates into phi.
static bool avx_int_accumulates(const SE_FGG_params* p)
{
    const int P = p->P;
    const int incrj = p->dims[2];
    const int incri = p->npdims[2] * p->dims[1];
    if ((P & 3) || (incri & 3) || (incrj & 3)) return false;
    if (P == 16 || P == 8 || P % 8 == 0) return false;
    return true;
}

static int do_base_gaussian(SE_FGG_work* w, const SE_FGG_params* p)
{
    if (!w || !valid_params(p) || !w->zs) return SE_ERR_INVALID;
    Stager s;
    const size_t P3 = (size_t)p->P * p->P * p->P;
    double* zs = (double*)s.use(w->zs, P3 * 8, false, true);
    SE_TRY(s.copy_in());
    k_base_gaussian<<<blocks(P3, 256), 256>>>(zs, to_dev(p));
    return s.finish();
}

static int do_expand(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p,
                     int periodicity, bool force)
{
    if (!w || !st || !valid_params(p)) return SE_ERR_INVALID;
    if (p->N == 0) return SE_OK;
    if (!st->x || !w->zx || !w->zy || !w->zz || !w->idx) return SE_ERR_INVALID;
    if (force && (!w->zfx || !w->zfy || !w->zfz)) return SE_ERR_INVALID;
    Stager s;
    const size_t NP = (size_t)p->N * p->P;
    const double* x = (const double*)s.use(st->x, 24 * (size_t)p->N, true, false);
    double* zx = (double*)s.use(w->zx, NP * 8, false, true);
    double* zy = (double*)s.use(w->zy, NP * 8, false, true);
    double* zz = (double*)s.use(w->zz, NP * 8, false, true);
    double* fx = force ? (double*)s.use(w->zfx, NP * 8, false, true) : nullptr;
    double* fy = force ? (double*)s.use(w->zfy, NP * 8, false, true) : nullptr;
    double* fz = force ? (double*)s.use(w->zfz, NP * 8, false, true) : nullptr;
    int* idx = (int*)s.use(w->idx, 4 * (size_t)p->N, false, true);
    SE_TRY(s.copy_in());
    k_expand_all<<<blocks(p->N, 128), 128>>>(to_dev(p), x, periodicity, zx, zy, zz, fx, fy, fz, idx);
    return s.finish();
}

static int do_grid_split(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p,
                         int force_order)
{
    if (!w || !st || !valid_params(p)) return SE_ERR_INVALID;
    if (p->N == 0) return SE_OK;
    if (!w->H || !w->zs || !w->zx || !w->zy || !w->zz || !w->idx || !st->q) return SE_ERR_INVALID;
    Stager s;
    const size_t NP = (size_t)p->N * p->P, P3 = (size_t)p->P * p->P * p->P;
    double* H = (double*)s.use(w->H, npad(p) * 8, true, true);
    const double* q = (const double*)s.use(st->q, 8 * (size_t)p->N, true, false);
    const double* zs = (const double*)s.use(w->zs, P3 * 8, true, false);
    const double* zx = (const double*)s.use(w->zx, NP * 8, true, false);
    const double* zy = (const double*)s.use(w->zy, NP * 8, true, false);
    const double* zz = (const double*)s.use(w->zz, NP * 8, true, false);
    const int* idx = (const int*)s.use(w->idx, 4 * (size_t)p->N, true, false);
    SE_TRY(s.copy_in());
    k_grid_split<<<p->N, 256>>>(H, q, zs, zx, zy, zz, idx, to_dev(p), force_order);
    return s.finish();
}

static int do_grid_vanilla(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    if (!w || !st || !valid_params(p)) return SE_ERR_INVALID;
    if (p->N == 0) return SE_OK;
    if (!w->H || !w->zs || !st->x || !st->q) return SE_ERR_INVALID;
    Stager s;
    const size_t P3 = (size_t)p->P * p->P * p->P;
    double* H = (double*)s.use(w->H, npad(p) * 8, true, true);
    const double* x = (const double*)s.use(st->x, 24 * (size_t)p->N, true, false);
    const double* q = (const double*)s.use(st->q, 8 * (size_t)p->N, true, false);
    const double* zs = (const double*)s.use(w->zs, P3 * 8, true, false);
    SE_TRY(s.copy_in());
    k_grid_vanilla<<<p->N, 256>>>(H, x, q, zs, to_dev(p), periodicity_default());
    return s.finish();
}

static int do_wrap(double* H_per, const SE_FGG_work* w, const SE_FGG_params* p, int periodicity)
{
    if (!H_per || !w || !w->H || !valid_params(p)) return SE_ERR_INVALID;
    const long long nout = nper_of(p, periodicity);
    Stager s;
    double* Hp = (double*)s.use(H_per, (size_t)nout * 8, true, true);
    const double* H = (const double*)s.use(w->H, npad(p) * 8, true, false);
    SE_TRY(s.copy_in());
    k_wrap<<<blocks(nout, 256), 256>>>(Hp, H, to_dev(p), periodicity, nout);
    return s.finish();
}

static int do_extend(SE_FGG_work* w, const double* H_per, const SE_FGG_params* p,
                     int periodicity)
{
    if (!H_per || !w || !w->H || !valid_params(p)) return SE_ERR_INVALID;
    const long long nin = nper_of(p, periodicity);
    Stager s;
    double* H = (double*)s.use(w->H, npad(p) * 8, false, true);
    const double* Hp = (const double*)s.use(H_per, (size_t)nin * 8, true, false);
    SE_TRY(s.copy_in());
    const int ph = periodicity == 3 ? p->P_half : ((p->P & 1) ? (p->P - 1) / 2 : p->P / 2);
    k_extend<<<blocks((long long)npad(p), 256), 256>>>(H, Hp, to_dev(p), periodicity, ph);
    return s.finish();
}

static int do_int_split(double* phi, const SE_FGG_work* w, const SE_FGG_params* p,
                        bool accumulate)
{
    if (!w || !valid_params(p)) return SE_ERR_INVALID;
    if (p->N == 0) return SE_OK;
    if (!phi || !w->H || !w->zs || !w->zx || !w->zy || !w->zz || !w->idx) return SE_ERR_INVALID;
    Stager s;
    const size_t NP = (size_t)p->N * p->P, P3 = (size_t)p->P * p->P * p->P;
    double* ph = (double*)s.use(phi, 8 * (size_t)p->N, accumulate, true);
    const double* H = (const double*)s.use(w->H, npad(p) * 8, true, false);
    const double* zs = (const double*)s.use(w->zs, P3 * 8, true, false);
    const double* zx = (const double*)s.use(w->zx, NP * 8, true, false);
    const double* zy = (const double*)s.use(w->zy, NP * 8, true, false);
    const double* zz = (const double*)s.use(w->zz, NP * 8, true, false);
    const int* idx = (const int*)s.use(w->idx, 4 * (size_t)p->N, true, false);
    SE_TRY(s.copy_in());
    const double h3 = p->h * p->h * p->h;
    k_int_split<<<blocks(p->N, 8), 256>>>(ph, H, zs, zx, zy, zz, idx, to_dev(p), h3, accumulate);
    return s.finish();
}

static int do_int_vanilla(double* phi, const SE_FGG_work* w, const SE_state* st,
                          const SE_FGG_params* p)
{
    if (!w || !st || !valid_params(p)) return SE_ERR_INVALID;
    if (p->N == 0) return SE_OK;
    if (!phi || !w->H || !w->zs || !st->x) return SE_ERR_INVALID;
    Stager s;
    const size_t P3 = (size_t)p->P * p->P * p->P;
    double* ph = (double*)s.use(phi, 8 * (size_t)p->N, false, true);
    const double* H = (const double*)s.use(w->H, npad(p) * 8, true, false);
    const double* x = (const double*)s.use(st->x, 24 * (size_t)p->N, true, false);
    const double* zs = (const double*)s.use(w->zs, P3 * 8, true, false);
    SE_TRY(s.copy_in());
    const double h3 = p->h * p->h * p->h;
    k_int_vanilla<<<blocks(p->N, 8), 256>>>(ph, H, x, zs, to_dev(p), periodicity_default(), h3);
    return s.finish();
}

static int do_int_split_force(double* force, const SE_state* st, const SE_FGG_work* w,
                              const SE_FGG_params* p)
{
    if (!w || !st || !valid_params(p)) return SE_ERR_INVALID;
    if (p->N == 0) return SE_OK;
    if (!force || !st->q || !w->H || !w->zs || !w->zx || !w->zy || !w->zz || !w->zfx ||
        !w->zfy || !w->zfz || !w->idx)
        return SE_ERR_INVALID;
    Stager s;
    const size_t NP = (size_t)p->N * p->P, P3 = (size_t)p->P * p->P * p->P;
    double* f = (double*)s.use(force, 24 * (size_t)p->N, false, true);
    const double* q = (const double*)s.use(st->q, 8 * (size_t)p->N, true, false);
    const double* H = (const double*)s.use(w->H, npad(p) * 8, true, false);
    const double* zs = (const double*)s.use(w->zs, P3 * 8, true, false);
    const double* zx = (const double*)s.use(w->zx, NP * 8, true, false);
    const double* zy = (const double*)s.use(w->zy, NP * 8, true, false);
    const double* zz = (const double*)s.use(w->zz, NP * 8, true, false);
    const double* fx = (const double*)s.use(w->zfx, NP * 8, true, false);
    const double* fy = (const double*)s.use(w->zfy, NP * 8, true, false);
    const double* fz = (const double*)s.use(w->zfz, NP * 8, true, false);
    const int* idx = (const int*)s.use(w->idx, 4 * (size_t)p->N, true, false);
    SE_TRY(s.copy_in());
    const double h3 = p->h * p->h * p->h;
    k_int_split_force<<<blocks(p->N, 8), 256>>>(f, q, H, zs, zx, zy, zz, fx, fy, fz, idx,
                                                 to_dev(p), h3);
    return s.finish();
}

static int do_int_force_vanilla(double* force, const SE_FGG_work* w, const SE_state* st,
                                const SE_FGG_params* p)
{
    if (!w || !st || !valid_params(p)) return SE_ERR_INVALID;
    if (p->N == 0) return SE_OK;
    if (!force || !w->H || !w->zs || !st->x || !st->q) return SE_ERR_INVALID;
    Stager s;
    const size_t P3 = (size_t)p->P * p->P * p->P;
    double* f = (double*)s.use(force, 24 * (size_t)p->N, false, true);
    const double* H = (const double*)s.use(w->H, npad(p) * 8, true, false);
    const double* x = (const double*)s.use(st->x, 24 * (size_t)p->N, true, false);
    const double* q = (const double*)s.use(st->q, 8 * (size_t)p->N, true, false);
    const double* zs = (const double*)s.use(w->zs, P3 * 8, true, false);
    SE_TRY(s.copy_in());
    const double h3 = p->h * p->h * p->h;
    k_int_force_vanilla<<<blocks(p->N, 4), 128>>>(f, H, x, q, zs, to_dev(p), h3);
    return s.finish();
}

// Managed arrays of the workspace and system allocators.  A caller that
// allocates and frees its workspace on every solve (spectral_ewald() does)
// would otherwise pay for a fresh managed allocation and its first touch on
// the device each time: freed arrays go to an idle pool (at most LIMIT bytes,
// largest freed first beyond that) and later allocations of a similar size
// take them back, zeroed again.
struct ManagedPool {
    std::mutex mu;
    std::unordered_map<void*, size_t> mine;   // every array this pool handed out
    std::multimap<size_t, void*> idle;
    size_t idle_bytes = 0;
    static constexpr size_t LIMIT = size_t(4) << 30;

    int take(void** p, size_t bytes)
    {
        {
            std::lock_guard<std::mutex> lock(mu);
            auto it = idle.lower_bound(bytes);
            if (it != idle.end() && it->first <= 2 * bytes) {
                *p = it->second;
                idle_bytes -= it->first;
                idle.erase(it);
                return SE_OK;
            }
        }
        SE_CUDA(cudaMallocManaged(p, bytes));
        std::lock_guard<std::mutex> lock(mu);
        mine[*p] = bytes;
        return SE_OK;
    }

    // false: not one of this pool's arrays
    bool give_back(void* p)
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = mine.find(p);
        if (it == mine.end()) return false;
        idle.emplace(it->second, p);
        idle_bytes += it->second;
        while (idle_bytes > LIMIT && !idle.empty()) {
            auto big = std::prev(idle.end());
            cudaFree(big->second);
            idle_bytes -= big->first;
            mine.erase(big->second);
            idle.erase(big);
        }
        return true;
    }
};

static ManagedPool& managed_pool()
{
    static ManagedPool* m = new ManagedPool();
    return *m;
}

static int managed_zeros(void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 8;
    SE_TRY(managed_pool().take(p, bytes));
    SE_CUDA(cudaMemset(*p, 0, bytes));
    SE_CUDA(cudaDeviceSynchronize());
    return SE_OK;
}

static void release(void* p)
{
    if (!p) return;
    if (managed_pool().give_back(p)) return;
    if (on_device(p)) cudaFree(p);
    else free(p);
}

static int do_allocate(SE_FGG_work* w, const SE_FGG_params* p, int zs, int expa, bool force)
{
    if (!w || !valid_params(p)) return SE_ERR_INVALID;
    memset(w, 0, sizeof(*w));
    const size_t NP = (size_t)p->N * p->P, P3 = (size_t)p->P * p->P * p->P;
    SE_TRY(managed_zeros((void**)&w->H, npad(p) * 8));
    if (zs) SE_TRY(managed_zeros((void**)&w->zs, P3 * 8));
    w->free_zs = zs;
    if (expa) {
        SE_TRY(managed_zeros((void**)&w->zx, NP * 8));
        SE_TRY(managed_zeros((void**)&w->zy, NP * 8));
        SE_TRY(managed_zeros((void**)&w->zz, NP * 8));
        SE_TRY(managed_zeros((void**)&w->idx, (size_t)p->N * 4));
        if (force) {
            SE_TRY(managed_zeros((void**)&w->zfx, NP * 8));
            SE_TRY(managed_zeros((void**)&w->zfy, NP * 8));
            SE_TRY(managed_zeros((void**)&w->zfz, NP * 8));
        }
    }
    w->free_fgg_expa = expa;
    return SE_OK;
}

}  // namespace legacy
}  // namespace se

using namespace se::legacy;

// ================================================================ ABI ====

extern "C" {

int is_odd(int p) { return p & 1; }
int isnot_div_by_4(int p) { return p & 3; }
int half(int p) { return (p & 1) ? (p - 1) / 2 : p / 2; }

int se_gpu_last_error(void) { return t_err; }
const char* se_gpu_last_error_string(void) { return t_msg; }

// ---- parameters ----
void SE_FGG_pack_params(SE_FGG_params* params, int N, int M0, int M1, int M2, int P, double c,
                        double h)
{
    params->N = N;
    params->P = P;
    params->P_half = half(P);
    params->c = c;
    params->d = pow(c / PI_D, 1.5);
    params->h = h;
    params->a = -1;
    params->b = -1;
    params->dims[0] = M0;
    params->dims[1] = M1;
    params->dims[2] = M2;
    params->npdims[0] = M0 + P;
    params->npdims[1] = M1 + P;
    params->npdims[2] = M2 + P;
}

void SE2P_FGG_pack_params(SE_FGG_params* params, int N, int M0, int M1, int M2, int P,
                          double c, double h, double a)
{
    SE_FGG_pack_params(params, N, M0, M1, M2, P, c, h);
    params->a = a;
}

void SE1P_FGG_pack_params(SE_FGG_params* params, int N, int M0, int M1, int M2, int P,
                          double c, double h, double a, double b)
{
    SE_FGG_pack_params(params, N, M0, M1, M2, P, c, h);
    params->a = a;
    params->b = b;
}

void parse_params(SE_opt* opt, double xi)
{
    const double h0 = opt->box[0] / (double)opt->M;
    const double w0 = (double)opt->P * h0 / 2.;
    const double r = 2.0 * w0 * xi / opt->m;
    const double eta0 = r * r;
    opt->h = h0;
    opt->c = 2.0 * xi * xi / eta0;
    opt->w = w0;
    opt->eta = eta0;
    opt->xi = xi;
}

void SE_FGG_FCN_params(SE_FGG_params* params, const SE_opt* opt, int N)
{
    params->N = N;
    params->P = (int)opt->P;
    params->P_half = half(opt->P);
    params->c = opt->c;
    params->d = pow(params->c / PI_D, 1.5);
    params->h = opt->box[0] / opt->M;
    params->a = -1.79769e+308;
    for (int d = 0; d < 3; d++) {
        params->dims[d] = opt->M;
        params->npdims[d] = opt->M + params->P;
    }
}

double SE_init_params(int* M, int* P, double* m, double eps, double L, double xi,
                      const double* q, int N)
{
    (void)eps;
    double Q = 0.;
    for (int i = 0; i < N; i++) Q += q[i] * q[i];
    const int iP = *P;
    const double ml = .95 * sqrt(PI_D * iP);
    const double k_inf = 2. * xi * L;
    int Ml = (int)ceil(2. * k_inf + 1) + 2;
    if (Ml < iP) Ml = iP;
    if (Ml % 4) Ml += 4 - Ml % 4;   // the AVX build (SE_general.c:559-562)
    *m = ml;
    *M = Ml;
    return Q;
}

// ---- workspace ----
void SE_FGG_allocate_workspace(SE_FGG_work* w, const SE_FGG_params* p, int zs, int expa)
{
    report(do_allocate(w, p, zs, expa, false), "SE_FGG_allocate_workspace");
}

void SE_FGG_allocate_workspace_SSE_force(SE_FGG_work* w, const SE_FGG_params* p, int zs,
                                         int expa)
{
    report(do_allocate(w, p, zs, expa, true), "SE_FGG_allocate_workspace_SSE_force");
}

double* SE_FGG_allocate_grid(const SE_FGG_params* p)
{
    void* g = nullptr;
    report(valid_params(p) ? managed_zeros(&g, nper(p) * 8) : SE_ERR_INVALID,
           "SE_FGG_allocate_grid");
    return (double*)g;
}

double* SE_FGG_allocate_vec(int n)
{
    void* g = nullptr;
    report(n >= 0 ? managed_zeros(&g, (size_t)n * 8) : SE_ERR_INVALID, "SE_FGG_allocate_vec");
    return (double*)g;
}

void SE_FGG_free_workspace(SE_FGG_work* w)
{
    release(w->H);
    if (w->free_zs) release(w->zs);
    if (w->free_fgg_expa) {
        release(w->zx);
        release(w->zy);
        release(w->zz);
        release(w->idx);
    }
}

void SE_FGG_free_workspace_SSE_force(SE_FGG_work* w)
{
    SE_FGG_free_workspace(w);
    if (w->free_fgg_expa) {
        release(w->zfx);
        release(w->zfy);
        release(w->zfz);
    }
}

// ---- systems (SE_fgg.c:266-322) ----
void SE_init_unit_system(SE_state* s, const SE_FGG_params* params)
{
    const int N = params->N;
    if (N % 2 != 0) return;
    if (managed_zeros((void**)&s->x, 24 * (size_t)N) || managed_zeros((void**)&s->q, 8 * (size_t)N) ||
        managed_zeros((void**)&s->phi, 8 * (size_t)N)) {
        report(SE_ERR_NOMEM, "SE_init_unit_system");
        return;
    }
    FILE* fp = fopen("atoms.txt", "r");
    if (!fp) {
        printf("Not successful!!!\n");
        return;
    }
    int err = 0;
    for (int i = 0; i < N; i++) {
        err = fscanf(fp, "%lf", &s->x[i]);
        err |= fscanf(fp, "%lf", &s->x[i + N]);
        err |= fscanf(fp, "%lf", &s->x[i + 2 * N]);
        err |= fscanf(fp, "%lf", &s->q[i]);
    }
    fclose(fp);
    if (err == EOF) printf("Not successful!!!\n");
}

void SE_init_system(SE_state* s, const SE_FGG_params* params)
{
    const int N = params->N;
    if (managed_zeros((void**)&s->x, 24 * (size_t)N) || managed_zeros((void**)&s->q, 8 * (size_t)N) ||
        managed_zeros((void**)&s->phi, 8 * (size_t)N)) {
        report(SE_ERR_NOMEM, "SE_init_system");
        return;
    }
    for (int i = 0; i < N; i++) {
        s->q[i] = -1 + 2 * ((double)rand() / RAND_MAX);
        s->x[i] = (double)rand() / RAND_MAX;
        s->x[i + N] = (double)rand() / RAND_MAX;
        s->x[i + 2 * N] = (double)rand() / RAND_MAX;
    }
}

void SE_free_system(SE_state* s)
{
    release(s->x);
    release(s->q);
}

// ---- utilities ----
double SE_gettime(void)
{
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int SE_prod3(const int v[3]) { return v[0] * v[1] * v[2]; }

void SE_fp_set_zero(double* x, int N)
{
    if (!x || N <= 0) return;
    if (on_device(x)) {
        cudaError_t e = cudaMemset(x, 0, sizeof(double) * (size_t)N);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        report(e == cudaSuccess ? SE_OK : SE_ERR_CUDA, "SE_fp_set_zero");
    } else {
        for (int i = 0; i < N; i++) x[i] = 0.0;
    }
}

double calc_energy(SE_state st, int N)
{
    if (N <= 0) return 0.0;
    Stager s;
    const double* phi = (const double*)s.use(st.phi, 8 * (size_t)N, true, false);
    const double* q = (const double*)s.use(st.q, 8 * (size_t)N, true, false);
    double* e = nullptr;
    double out = 0.0;
    int r = s.copy_in();
    if (r == SE_OK) r = cudaMalloc(&e, sizeof(double)) == cudaSuccess ? SE_OK : SE_ERR_NOMEM;
    if (r == SE_OK) r = se_energy(phi, q, N, e, nullptr);
    if (r == SE_OK) r = s.finish();
    if (r == SE_OK)
        r = cudaMemcpy(&out, e, sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess ? SE_OK
                                                                                       : SE_ERR_CUDA;
    if (e) cudaFree(e);
    report(r, "calc_energy");
    return out;
}

void SE_FGG_reorder_system(SE_state* st, const SE_FGG_work* w, const SE_FGG_params* p)
{
    int r = SE_OK;
    if (!st || !w || !valid_params(p) || !w->idx || !st->x || !st->q) r = SE_ERR_INVALID;
    const int N = p ? p->N : 0;
    if (r == SE_OK && N > 0) {
        // key range of the padded grid indices
        std::vector<int> hidx(N);
        Stager s;
        int* idx = (int*)s.use(w->idx, 4 * (size_t)N, true, false);
        double* x = (double*)s.use(st->x, 24 * (size_t)N, true, true);
        double* q = (double*)s.use(st->q, 8 * (size_t)N, true, true);
        r = s.copy_in();
        if (r == SE_OK)
            r = cudaMemcpy(hidx.data(), idx, 4 * (size_t)N, cudaMemcpyDeviceToHost) == cudaSuccess
                    ? SE_OK : SE_ERR_CUDA;
        int lo = 0, hi = 0;
        if (r == SE_OK) {
            lo = *std::min_element(hidx.begin(), hidx.end());
            hi = *std::max_element(hidx.begin(), hidx.end());
        }
        const int nkeys = hi - lo + 1;
        void* scratch = nullptr;
        int *keys = nullptr, *perm = nullptr;
        double *xc = nullptr, *qc = nullptr;
        const size_t sb = se::sort_scratch_bytes(N, nkeys);
        if (r == SE_OK &&
            (cudaMalloc(&scratch, sb) != cudaSuccess || cudaMalloc(&keys, 4 * (size_t)N) != cudaSuccess ||
             cudaMalloc(&perm, 4 * (size_t)N) != cudaSuccess ||
             cudaMalloc(&xc, 24 * (size_t)N) != cudaSuccess || cudaMalloc(&qc, 8 * (size_t)N) != cudaSuccess))
            r = SE_ERR_NOMEM;
        if (r == SE_OK) {
            k_key_shift<<<blocks(N, 256), 256>>>(idx, keys, N, lo);
            r = se::stable_sort(keys, nullptr, N, nkeys, perm, nullptr, nullptr, scratch, sb,
                                nullptr, nullptr);
        }
        if (r == SE_OK) {
            cudaMemcpy(xc, x, 24 * (size_t)N, cudaMemcpyDeviceToDevice);
            cudaMemcpy(qc, q, 8 * (size_t)N, cudaMemcpyDeviceToDevice);
            k_permute_state<<<blocks(N, 256), 256>>>(x, q, xc, qc, perm, N);
            r = s.finish();
        }
        cudaFree(scratch);
        cudaFree(keys);
        cudaFree(perm);
        cudaFree(xc);
        cudaFree(qc);
    }
    report(r, "SE_FGG_reorder_system");
}

// ---- base Gaussian, expansion ----
void SE_FGG_base_gaussian(SE_FGG_work* w, const SE_FGG_params* p)
{
    report(do_base_gaussian(w, p), "SE_FGG_base_gaussian");
}

void SE_FGG_expand_all(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    report(do_expand(w, st, p, periodicity_default(), false), "SE_FGG_expand_all");
}

void SE3P_FGG_expand_all(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    report(do_expand(w, st, p, 3, false), "SE3P_FGG_expand_all");
}

void SE2P_FGG_expand_all(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    report(do_expand(w, st, p, 2, false), "SE2P_FGG_expand_all");
}

void SE1P_FGG_expand_all(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    report(do_expand(w, st, p, 1, false), "SE1P_FGG_expand_all");
}

void SE_FGG_expand_all_SSE_force(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    report(do_expand(w, st, p, 3, true), "SE_FGG_expand_all_SSE_force");
}

// ---- spread ----
void SE_FGG_grid(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    report(do_grid_vanilla(w, st, p), "SE_FGG_grid");
}

#define SE_GRID_POT(name) \
    void name(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p) \
    { report(do_grid_split(w, st, p, 0), #name); }
#define SE_GRID_FORCE(name) \
    void name(SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p) \
    { report(do_grid_split(w, st, p, 1), #name); }

SE_GRID_POT(SE_FGG_grid_split)
SE_GRID_POT(SE_FGG_grid_split_SSE_dispatch)
SE_GRID_POT(SE_FGG_grid_split_SSE)
SE_GRID_POT(SE_FGG_grid_split_SSE_u8)
SE_GRID_POT(SE_FGG_grid_split_SSE_P16)
SE_GRID_POT(SE_FGG_grid_split_AVX_dispatch)
SE_GRID_POT(SE_FGG_grid_split_AVX)
SE_GRID_POT(SE_FGG_grid_split_AVX_P16)
SE_GRID_POT(SE_FGG_grid_split_AVX_P8)
SE_GRID_POT(SE_FGG_grid_split_AVX_u8)
SE_GRID_FORCE(SE_FGG_grid_split_force)
SE_GRID_FORCE(SE_FGG_grid_split_SSE_dispatch_force)
SE_GRID_FORCE(SE_FGG_grid_split_SSE_force)
SE_GRID_FORCE(SE_FGG_grid_split_SSE_u8_force)
SE_GRID_FORCE(SE_FGG_grid_split_SSE_P16_force)
SE_GRID_FORCE(SE_FGG_grid_split_AVX_dispatch_force)
SE_GRID_FORCE(SE_FGG_grid_split_AVX_P16_force)
SE_GRID_FORCE(SE_FGG_grid_split_AVX_P8_force)
SE_GRID_FORCE(SE_FGG_grid_split_AVX_u8_force)
SE_GRID_FORCE(SE_FGG_grid_split_AVX_force)

// ---- fold / unfold ----
void SE_FGG_wrap_fcn(double* H_per, const SE_FGG_work* w, const SE_FGG_params* p)
{
    report(do_wrap(H_per, w, p, 3), "SE_FGG_wrap_fcn");
}

void SE2P_FGG_wrap_fcn(double* H_per, const SE_FGG_work* w, const SE_FGG_params* p)
{
    report(do_wrap(H_per, w, p, 2), "SE2P_FGG_wrap_fcn");
}

void SE1P_FGG_wrap_fcn(double* H_per, const SE_FGG_work* w, const SE_FGG_params* p)
{
    report(do_wrap(H_per, w, p, 1), "SE1P_FGG_wrap_fcn");
}

void SE_FGG_extend_fcn(SE_FGG_work* w, const double* H_per, const SE_FGG_params* p)
{
    report(do_extend(w, H_per, p, 3), "SE_FGG_extend_fcn");
}

void SE2P_FGG_extend_fcn(SE_FGG_work* w, const double* H_per, const SE_FGG_params* p)
{
    report(do_extend(w, H_per, p, 2), "SE2P_FGG_extend_fcn");
}

void SE1P_FGG_extend_fcn(SE_FGG_work* w, const double* H_per, const SE_FGG_params* p)
{
    report(do_extend(w, H_per, p, 1), "SE1P_FGG_extend_fcn");
}

// ---- interpolate, POTENTIAL ----
void SE_FGG_int(double* phi, const SE_FGG_work* w, const SE_state* st, const SE_FGG_params* p)
{
    report(do_int_vanilla(phi, w, st, p), "SE_FGG_int");
}

#define SE_INT_POT(name, acc) \
    void name(double* phi, const SE_FGG_work* w, const SE_FGG_params* p) \
    { report(do_int_split(phi, w, p, acc), #name); }

SE_INT_POT(SE_FGG_int_split, false)
SE_INT_POT(SE_FGG_int_split_SSE_dispatch, false)
SE_INT_POT(SE_FGG_int_split_SSE, false)
SE_INT_POT(SE_FGG_int_split_SSE_u8, false)
SE_INT_POT(SE_FGG_int_split_SSE_P8, false)
SE_INT_POT(SE_FGG_int_split_SSE_P16, false)
SE_INT_POT(SE_FGG_int_split_AVX, true)
SE_INT_POT(SE_FGG_int_split_AVX_P8, false)
SE_INT_POT(SE_FGG_int_split_AVX_P16, false)
SE_INT_POT(SE_FGG_int_split_AVX_u8, false)

void SE_FGG_int_split_AVX_dispatch(double* phi, const SE_FGG_work* w, const SE_FGG_params* p)
{
    report(valid_params(p) ? do_int_split(phi, w, p, avx_int_accumulates(p)) : SE_ERR_INVALID,
           "SE_FGG_int_split_AVX_dispatch");
}

// ---- interpolate, FORCE ----
void SE_FGG_int_force(double* force, const SE_FGG_work* w, SE_state* st, const SE_FGG_params* p)
{
    report(do_int_force_vanilla(force, w, st, p), "SE_FGG_int_force");
}

#define SE_INT_FORCE(name) \
    void name(double* force, SE_state* st, const SE_FGG_work* w, const SE_FGG_params* p) \
    { report(do_int_split_force(force, st, w, p), #name); }

SE_INT_FORCE(SE_FGG_int_split_force)
SE_INT_FORCE(SE_FGG_int_split_SSE_dispatch_force)
SE_INT_FORCE(SE_FGG_int_split_SSE_force)
SE_INT_FORCE(SE_FGG_int_split_SSE_P8_force)
SE_INT_FORCE(SE_FGG_int_split_SSE_u8_force)
SE_INT_FORCE(SE_FGG_int_split_SSE_P16_force)
SE_INT_FORCE(SE_FGG_int_split_AVX_dispatch_force)
SE_INT_FORCE(SE_FGG_int_split_AVX_P16_force)
SE_INT_FORCE(SE_FGG_int_split_AVX_P8_force)
SE_INT_FORCE(SE_FGG_int_split_AVX_u8_force)
SE_INT_FORCE(SE_FGG_int_split_AVX_force)

// ---- k-space (SE_general.c) ----
void k_vec(int M, double* box, double* k1, double* k2, double* k3)
{
    double* k[3] = {k1, k2, k3};
    const int npos = (M % 2 == 0) ? M / 2 : (M - 1) / 2 + 1;
    for (int d = 0; d < 3; d++) {
        const double f = 2.0 * PI_D / box[d];
        for (int i = 0; i < M; i++) k[d][i] = f * (double)(i < npos ? i : i - M);
    }
}

void scaling(double scalar, double* Z, int n1, int n2, int n3, double* box)
{
    int r = (Z && n1 > 0 && n2 > 0 && n3 > 0 && box) ? SE_OK : SE_ERR_INVALID;
    if (r == SE_OK) {
        const long long n = (long long)n1 * n2 * n3;
        Stager s;
        double* z = (double*)s.use(Z, (size_t)n * 8, false, true);
        r = s.copy_in();
        if (r == SE_OK) {
            k_scaling<<<blocks(n, 256), 256>>>(z, n1, n2, n3, 2.0 * PI_D / box[0],
                                               2.0 * PI_D / box[1], 2.0 * PI_D / box[2], scalar);
            r = s.finish();
        }
    }
    report(r, "scaling");
}

void product_rc(t_complex* a, double* b, t_complex* c, int n1, int n2, int n3, int flag)
{
    int r = (a && b && c) ? SE_OK : SE_ERR_INVALID;
    const long long n = (long long)n1 * n2 * n3;
    if (r == SE_OK && n > 0) {
        Stager s;
        double2* dc = (double2*)s.use(c, (size_t)n * 16, c == a, true);
        const double2* da = (const double2*)s.use(a, (size_t)n * 16, true, false);
        const double* db = (const double*)s.use(b, (size_t)n * 8, true, false);
        r = s.copy_in();
        if (r == SE_OK) {
            k_product_rc<<<blocks(n, 256), 256>>>(dc, da, db, n, flag);
            r = s.finish();
        }
    }
    report(r, "product_rc");
}

void copy_r2c(double* in, t_complex* out, int n)
{
    int r = (in && out) ? SE_OK : SE_ERR_INVALID;
    if (r == SE_OK && n > 0) {
        Stager s;
        const double* di = (const double*)s.use(in, (size_t)n * 8, true, false);
        double2* dout = (double2*)s.use(out, (size_t)n * 16, false, true);
        r = s.copy_in();
        if (r == SE_OK) {
            k_copy_r2c<<<blocks(n, 256), 256>>>(di, dout, n);
            r = s.finish();
        }
    }
    report(r, "copy_r2c");
}

void copy_c2r(t_complex* in, double* out, int n)
{
    int r = (in && out) ? SE_OK : SE_ERR_INVALID;
    if (r == SE_OK && n > 0) {
        Stager s;
        const double2* di = (const double2*)s.use(in, (size_t)n * 16, true, false);
        double* dout = (double*)s.use(out, (size_t)n * 8, false, true);
        r = s.copy_in();
        if (r == SE_OK) {
            k_copy_c2r<<<blocks(n, 256), 256>>>(di, dout, n);
            r = s.finish();
        }
    }
    report(r, "copy_c2r");
}

// SE_general.c:204-230
void SE_fgg_int_force(double* x, double* q, double* H, int N, SE_opt opt, double* force_out)
{
    SE_FGG_params params;
    SE_FGG_FCN_params(&params, &opt, N);
    SE_FGG_work work;
    SE_FGG_allocate_workspace(&work, &params, 1, 0);
    if (t_err) return;
    SE_state st;
    st.x = x;
    st.q = q;
    st.phi = nullptr;
    SE_FGG_base_gaussian(&work, &params);
    if (!t_err) SE_FGG_extend_fcn(&work, H, &params);
    if (!t_err) SE_FGG_int_force(force_out, &work, &st, &params);
    const int saved = t_err;
    SE_FGG_free_workspace(&work);
    t_err = saved;
}

}  // extern "C"
