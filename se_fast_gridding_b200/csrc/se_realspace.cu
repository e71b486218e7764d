// se_realspace.cu -- the real-space and self terms of the Ewald sum beside
// the k-space solve: SE3P_direct_real_rc (SE_direct.c:464-506),
// SE3P_direct_real (:508-549) and SE3P_direct_self (:551-562), plus the
// real-space force (the gradient of the same sum; the reference has none).
//
// Two algorithms, chosen by the cutoff:
//   all pairs   any rc and layers: one thread per target, the sources in
//               tiles of 128 through shared memory, the images in the
//               reference's (p0, p1, p2) order -- the reference's summation
//               order for every target;
//   cell list   0 < rc <= L/2 with at least 3 cells of edge >= rc per axis:
//               particles sorted by cell (the library's stable sort), one
//               thread per target (in cell order) over the 27 neighbour cells.
//               Each particle keeps its position wrapped into the box and the
//               number of boxes it was moved by, so the image of a pair is
//               recovered exactly and the reference's limit |p| <= layers on
//               it holds for positions anywhere.
// Scratch memory of the cell list is taken from the stream-ordered pool
// (cudaMallocAsync) and returned on the same stream.
#include <cmath>

#include "se_internal.h"

namespace se {
namespace {

constexpr int RS_THREADS = 128;
constexpr double RS_PI = 3.14159265358979323846;

struct RsParams {
    int N, layers;
    double L, xi, rc, rc2, g;   // g = 2 xi / sqrt(pi)
};

// One pair term at separation d (|d|^2 = rr): potential and force weights.
template <bool FORCE>
__device__ __forceinline__ void pair_term(const RsParams& S, double qn, const double d[3],
                                          double rr, double& phi, double f[3])
{
    const double r = sqrt(rr);
    const double e = erfc(S.xi * r) / r;
    phi += qn * e;
    if (FORCE) {
        const double s = qn * (e + S.g * exp(-S.xi * S.xi * rr)) / rr;
        f[0] += s * d[0];
        f[1] += s * d[1];
        f[2] += s * d[2];
    }
}

template <bool FORCE>
__global__ void __launch_bounds__(RS_THREADS) k_real_allpairs(
    RsParams S, const double* __restrict__ x, const double* __restrict__ q,
    double* __restrict__ phi, double* __restrict__ force)
{
    __shared__ double4 src[RS_THREADS];
    const int N = S.N;
    const int m = blockIdx.x * RS_THREADS + threadIdx.x;
    double xm[3] = {0, 0, 0};
    if (m < N) {
        xm[0] = x[m];
        xm[1] = x[m + N];
        xm[2] = x[m + 2 * N];
    }
    double acc = 0, f[3] = {0, 0, 0};
    const int l = S.layers;
    for (int t0 = 0; t0 < N; t0 += RS_THREADS) {
        const int n = t0 + threadIdx.x;
        __syncthreads();
        if (n < N) src[threadIdx.x] = make_double4(x[n], x[n + N], x[n + 2 * N], q[n]);
        __syncthreads();
        if (m >= N) continue;
        const int cnt = min(RS_THREADS, N - t0);
        for (int j = 0; j < cnt; j++) {
            const double4 s = src[j];
            const double r0 = xm[0] - s.x, r1 = xm[1] - s.y, r2 = xm[2] - s.z;
            for (int p0 = -l; p0 <= l; p0++)
                for (int p1 = -l; p1 <= l; p1++)
                    for (int p2 = -l; p2 <= l; p2++) {
                        if (m == t0 + j && p0 == 0 && p1 == 0 && p2 == 0) continue;
                        const double d[3] = {r0 + p0 * S.L, r1 + p1 * S.L, r2 + p2 * S.L};
                        const double rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                        if (S.rc > 0 && rr > S.rc2) continue;
                        pair_term<FORCE>(S, s.w, d, rr, acc, f);
                    }
        }
    }
    if (m >= N) return;
    if (phi) phi[m] += acc;
    if (FORCE) {
        const double qm = q[m];
        force[m] += qm * f[0];
        force[m + N] += qm * f[1];
        force[m + 2 * N] += qm * f[2];
    }
}

// Cell of every particle (edge cs = L / nc >= rc), from its position wrapped
// into [0, L); the number of boxes it was moved by, packed per axis.
__global__ void k_real_keys(RsParams S, int nc, const double* __restrict__ x,
                            int* __restrict__ key)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= S.N) return;
    int c[3];
    for (int a = 0; a < 3; a++) {
        const double v = x[n + (long long)a * S.N];
        const double w = v - S.L * floor(v / S.L);
        c[a] = min((int)(w * nc / S.L), nc - 1);
    }
    key[n] = (c[0] * nc + c[1]) * nc + c[2];
}

// Sorted records: wrapped position and charge, and the box shifts k_a =
// floor(x_a / L) (each within +-511).
__global__ void k_real_gather(RsParams S, const int* __restrict__ perm,
                              const double* __restrict__ x, const double* __restrict__ q,
                              double4* __restrict__ rec, int* __restrict__ kbox)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.N) return;
    const int n = perm[s];
    double w[3];
    int k[3];
    for (int a = 0; a < 3; a++) {
        const double v = x[n + (long long)a * S.N];
        const double fl = floor(v / S.L);
        w[a] = v - S.L * fl;
        k[a] = (int)fl;
    }
    rec[s] = make_double4(w[0], w[1], w[2], q[n]);
    kbox[s] = ((k[0] + 512) & 1023) | (((k[1] + 512) & 1023) << 10) | (((k[2] + 512) & 1023) << 20);
}

__device__ __forceinline__ int kbox_of(int pk, int a) { return ((pk >> (10 * a)) & 1023) - 512; }

template <bool FORCE>
__global__ void __launch_bounds__(RS_THREADS) k_real_cells(
    RsParams S, int nc, const double4* __restrict__ rec, const int* __restrict__ kbox,
    const int* __restrict__ perm, const int* __restrict__ cell_off, const double* __restrict__ q,
    double* __restrict__ phi, double* __restrict__ force)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S.N) return;
    const double4 me = rec[s];
    const int km = kbox[s];
    const double xm[3] = {me.x, me.y, me.z};
    int c[3];
    for (int a = 0; a < 3; a++) c[a] = min((int)(xm[a] * nc / S.L), nc - 1);
    double acc = 0, f[3] = {0, 0, 0};
    for (int dx = -1; dx <= 1; dx++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dz = -1; dz <= 1; dz++) {
                const int cc[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
                int w[3], sh[3];   // wrapped neighbour cell and its box shift
                for (int a = 0; a < 3; a++) {
                    sh[a] = cc[a] < 0 ? -1 : (cc[a] >= nc ? 1 : 0);
                    w[a] = cc[a] - sh[a] * nc;
                }
                const int cell = (w[0] * nc + w[1]) * nc + w[2];
                for (int t = cell_off[cell]; t < cell_off[cell + 1]; t++) {
                    if (t == s && dx == 0 && dy == 0 && dz == 0) continue;
                    const double4 o = rec[t];
                    const double d[3] = {xm[0] - (o.x + sh[0] * S.L), xm[1] - (o.y + sh[1] * S.L),
                                         xm[2] - (o.z + sh[2] * S.L)};
                    const double rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                    if (rr > S.rc2) continue;
                    // the image index of the pair in raw coordinates
                    const int kt = kbox[t];
                    bool in = true;
                    for (int a = 0; a < 3; a++) {
                        const int p = kbox_of(kt, a) - kbox_of(km, a) - sh[a];
                        in = in && p >= -S.layers && p <= S.layers;
                    }
                    if (in) pair_term<FORCE>(S, o.w, d, rr, acc, f);
                }
            }
    const int m = perm[s];
    if (phi) phi[m] += acc;
    if (FORCE) {
        const double qm = me.w;
        force[m] += qm * f[0];
        force[m + S.N] += qm * f[1];
        force[m + 2 * S.N] += qm * f[2];
    }
}

__global__ void k_self(const double* __restrict__ q, int N, double c, double* __restrict__ phi)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < N) phi[m] -= c * q[m];
}

// Cells per axis of the cell-list form, or 0 when the all-pairs form applies.
int cells_per_axis(double L, double rc)
{
    if (!(rc > 0) || 2 * rc > L) return 0;
    const double nc = floor(L / rc);
    return (nc >= 3 && nc <= 256) ? (int)nc : 0;
}

int real_space(const double* x, const double* q, int N, double L, double xi, int layers,
               double rc, double* phi, double* force, cudaStream_t st)
{
    RsParams S;
    S.N = N;
    S.layers = layers;
    S.L = L;
    S.xi = xi;
    S.rc = rc > 0 ? rc : 0.0;
    S.rc2 = S.rc * S.rc;
    S.g = 2.0 * xi / sqrt(RS_PI);
    const int nc = cells_per_axis(L, rc);
    const unsigned nb = ceil_div(N, RS_THREADS);
    if (nc == 0) {
        if (force) k_real_allpairs<true><<<nb, RS_THREADS, 0, st>>>(S, x, q, phi, force);
        else k_real_allpairs<false><<<nb, RS_THREADS, 0, st>>>(S, x, q, phi, nullptr);
        SE_CUDA(cudaGetLastError());
        return SE_OK;
    }
    const int ncell = nc * nc * nc;
    const size_t sb = sort_scratch_bytes(N, ncell);
    const size_t nbytes = 256 * ((sizeof(int) * N + 255) / 256);
    const size_t rbytes = 256 * ((sizeof(double4) * N + 255) / 256);
    const size_t obytes = 256 * ((sizeof(int) * (ncell + 1) + 255) / 256);
    const size_t total = 3 * nbytes + rbytes + obytes + sb;
    char* base = nullptr;
    SE_CUDA(cudaMallocAsync((void**)&base, total, st));
    int* key = reinterpret_cast<int*>(base);
    int* perm = reinterpret_cast<int*>(base + nbytes);
    int* kbox = reinterpret_cast<int*>(base + 2 * nbytes);
    double4* rec = reinterpret_cast<double4*>(base + 3 * nbytes);
    int* off = reinterpret_cast<int*>(base + 3 * nbytes + rbytes);
    void* scratch = base + 3 * nbytes + rbytes + obytes;
    int r = SE_OK;
    k_real_keys<<<ceil_div(N, 256), 256, 0, st>>>(S, nc, x, key);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        r = stable_sort(key, nullptr, N, ncell, perm, nullptr, off, scratch, sb, st, nullptr);
        if (r == SE_OK) {
            k_real_gather<<<ceil_div(N, 256), 256, 0, st>>>(S, perm, x, q, rec, kbox);
            if (force)
                k_real_cells<true><<<nb, RS_THREADS, 0, st>>>(S, nc, rec, kbox, perm, off, q, phi,
                                                              force);
            else
                k_real_cells<false><<<nb, RS_THREADS, 0, st>>>(S, nc, rec, kbox, perm, off, q, phi,
                                                               nullptr);
            e = cudaGetLastError();
        }
    }
    cudaFreeAsync(base, st);
    if (e != cudaSuccess) return cuda_fail(e, "real-space kernels", __FILE__, __LINE__);
    return r;
}

}  // namespace
}  // namespace se

extern "C" int se_real_space(const double* x, const double* q, int N, double L, double xi,
                             int layers, double rc, double* phi, double* force, void* stream)
{
    if (N < 0 || !(L > 0) || !(xi > 0) || layers < 0 || layers > 64 || (!phi && !force) ||
        (N > 0 && (!x || !q)))
        return SE_ERR_INVALID;
    if (N == 0) return SE_OK;
    return se::real_space(x, q, N, L, xi, layers, rc, phi, force, se::as_stream(stream));
}

extern "C" int se_self_term(const double* q, int N, double xi, double* phi, void* stream)
{
    if (N < 0 || !(xi > 0) || (N > 0 && (!q || !phi))) return SE_ERR_INVALID;
    if (N == 0) return SE_OK;
    se::k_self<<<se::ceil_div(N, 256), 256, 0, se::as_stream(stream)>>>(
        q, N, 2.0 * xi / sqrt(se::RS_PI), phi);
    SE_CUDA(cudaGetLastError());
    return SE_OK;
}
