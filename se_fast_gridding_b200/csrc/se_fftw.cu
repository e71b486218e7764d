// se_fftw.cu -- the FFTW 3 subset of include/fftw3.h on cuFFT.
//
// SE_fast_gridding calls FFTW for its k-space step (spectral_ewald.c:80,
// 119-123,133,178-179; SE_general.c:234-270).  Plans here wrap cuFFT plans of
// the same shape and kind; fftw_execute transforms the plan's arrays on the
// GPU (host arrays are staged through device memory, managed/device arrays
// are used in place).  fftw_malloc returns CUDA managed memory so that arrays
// allocated through it are transformed without copies.
//
// The caller plans and destroys its transforms on every solve
// (spectral_ewald.c:101-102,159-160), and a cuFFT plan of a 128^3 grid takes
// ~12 ms to make: fftw_destroy_plan keeps the cuFFT plan and its device
// staging buffers (up to PLAN_CACHE per shape, kind and device) for the next
// fftw_plan_* of the same shape and kind.
#include <cufft.h>

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "fftw3.h"
#include "se_fgg_gpu.h"
#include "se_internal.h"

namespace {

enum { K_C2C, K_R2C, K_C2R };

bool on_device(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// A cuFFT plan and the device staging buffers of its host arrays.
struct Cached {
    cufftHandle h;
    void* din;
    void* dout;
    size_t din_cap, dout_cap;
};
constexpr size_t PLAN_CACHE = 4;
using PlanKey = std::tuple<int, int, int, int, int>;   // device, n0, n1, n2, kind
std::mutex g_plan_mu;

std::map<PlanKey, std::vector<Cached>>& plan_cache()
{
    static auto* m = new std::map<PlanKey, std::vector<Cached>>();
    return *m;
}

}  // namespace

struct fftw_plan_s {
    int n[3];
    int kind;
    int sign;
    void* in;
    void* out;
    cufftHandle h;
    void* din;    // device staging (host arrays only)
    void* dout;
    size_t din_cap, dout_cap;
    size_t in_bytes, out_bytes;
    int dev;
};

static fftw_plan make_plan(int n0, int n1, int n2, int kind, int sign, void* in, void* out)
{
    if (n0 < 1 || n1 < 1 || n2 < 1) return nullptr;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->n[0] = n0;
    p->n[1] = n1;
    p->n[2] = n2;
    p->kind = kind;
    p->sign = sign;
    p->in = in;
    p->out = out;
    const size_t nr = (size_t)n0 * n1 * n2, nh = (size_t)n0 * n1 * (n2 / 2 + 1);
    cufftType t = kind == K_C2C ? CUFFT_Z2Z : kind == K_R2C ? CUFFT_D2Z : CUFFT_Z2D;
    p->in_bytes = kind == K_C2C ? nr * 16 : kind == K_R2C ? nr * 8 : nh * 16;
    p->out_bytes = kind == K_C2C ? nr * 16 : kind == K_R2C ? nh * 16 : nr * 8;
    if (cudaGetDevice(&p->dev) != cudaSuccess) {
        free(p);
        return nullptr;
    }
    {
        std::lock_guard<std::mutex> lock(g_plan_mu);
        auto it = plan_cache().find(PlanKey(p->dev, n0, n1, n2, kind));
        if (it != plan_cache().end() && !it->second.empty()) {
            const Cached c = it->second.back();
            it->second.pop_back();
            p->h = c.h;
            p->din = c.din;
            p->dout = c.dout;
            p->din_cap = c.din_cap;
            p->dout_cap = c.dout_cap;
            return p;
        }
    }
    if (cufftPlan3d(&p->h, n0, n1, n2, t) != CUFFT_SUCCESS) {
        fprintf(stderr, "[se_gpu] cufftPlan3d(%d,%d,%d) failed\n", n0, n1, n2);
        free(p);
        return nullptr;
    }
    return p;
}

extern "C" {

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags)
{
    (void)flags;
    return make_plan(n0, n1, n2, K_C2C, sign, in, out);
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out,
                               unsigned flags)
{
    (void)flags;
    return make_plan(n0, n1, n2, K_R2C, FFTW_FORWARD, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out,
                               unsigned flags)
{
    (void)flags;
    return make_plan(n0, n1, n2, K_C2R, FFTW_BACKWARD, in, out);
}

void fftw_execute(const fftw_plan p)
{
    if (!p) return;
    const bool hin = !on_device(p->in), hout = !on_device(p->out);
    const bool inplace = p->in == p->out;
    const size_t big = p->in_bytes > p->out_bytes ? p->in_bytes : p->out_bytes;
    void* din = p->in;
    void* dout = p->out;
    cudaError_t e = cudaSuccess;
    auto reserve = [&](void** buf, size_t* cap, size_t bytes) {
        if (e != cudaSuccess || (*buf && *cap >= bytes)) return;
        if (*buf) cudaFree(*buf);
        *buf = nullptr;
        *cap = 0;
        e = cudaMalloc(buf, bytes);
        if (e == cudaSuccess) *cap = bytes;
    };
    if (hin || hout) {
        reserve(&p->din, &p->din_cap, inplace ? big : p->in_bytes);
        if (!inplace) reserve(&p->dout, &p->dout_cap, p->out_bytes);
    }
    if (hin) din = p->din;
    if (hout) dout = inplace ? din : p->dout;
    if (inplace && (hin != hout)) dout = din;   // mixed kinds cannot alias
    // an in-place real transform uses FFTW's (and cuFFT's) padded layout:
    // n0 x n1 x 2(n2/2 + 1) reals, the size of the half spectrum, both ways
    const size_t in_copy = inplace ? big : p->in_bytes, out_copy = inplace ? big : p->out_bytes;
    int staged = SE_OK;
    if (e == cudaSuccess && hin) staged = se::host_to_device(din, p->in, in_copy);
    cufftResult r = CUFFT_SUCCESS;
    if (e == cudaSuccess && staged == SE_OK) {
        cufftSetStream(p->h, 0);
        if (p->kind == K_C2C)
            r = cufftExecZ2Z(p->h, (cufftDoubleComplex*)din, (cufftDoubleComplex*)dout,
                             p->sign == FFTW_FORWARD ? CUFFT_FORWARD : CUFFT_INVERSE);
        else if (p->kind == K_R2C)
            r = cufftExecD2Z(p->h, (cufftDoubleReal*)din, (cufftDoubleComplex*)dout);
        else
            r = cufftExecZ2D(p->h, (cufftDoubleComplex*)din, (cufftDoubleReal*)dout);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && staged == SE_OK && hout)
        staged = se::device_to_host(p->out, dout, out_copy);
    if (e != cudaSuccess || r != CUFFT_SUCCESS || staged != SE_OK)
        fprintf(stderr, "[se_gpu] fftw_execute failed: %s / cuFFT %d / staging %d\n",
                cudaGetErrorString(e), (int)r, staged);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lock(g_plan_mu);
        auto& v = plan_cache()[PlanKey(p->dev, p->n[0], p->n[1], p->n[2], p->kind)];
        if (v.size() < PLAN_CACHE) {
            v.push_back(Cached{p->h, p->din, p->dout, p->din_cap, p->dout_cap});
            free(p);
            return;
        }
    }
    cufftDestroy(p->h);
    if (p->din) cudaFree(p->din);
    if (p->dout) cudaFree(p->dout);
    free(p);
}

void* fftw_malloc(size_t n)
{
    void* p = nullptr;
    if (cudaMallocManaged(&p, n ? n : 1) != cudaSuccess) return nullptr;
    return p;
}

void fftw_free(void* p)
{
    if (!p) return;
    if (on_device(p)) cudaFree(p);
    else free(p);
}

void fftw_cleanup(void) {}

// SE_general.c:234-270: one-shot transforms through the plans above
void do_fft_r2c_3d(double* in, t_complex* out, int n1, int n2, int n3)
{
    fftw_plan p = fftw_plan_dft_r2c_3d(n1, n2, n3, in, out, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
}

void do_fft_c2r_3d(t_complex* in, double* out, int n1, int n2, int n3)
{
    fftw_plan p = fftw_plan_dft_c2r_3d(n1, n2, n3, in, out, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
}

void do_fft_c2c_forward_3d(t_complex* in, t_complex* out, int n1, int n2, int n3)
{
    fftw_plan p = fftw_plan_dft_3d(n1, n2, n3, in, out, FFTW_FORWARD, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
}

void do_fft_c2c_backward_3d(t_complex* in, t_complex* out, int n1, int n2, int n3)
{
    fftw_plan p = fftw_plan_dft_3d(n1, n2, n3, in, out, FFTW_BACKWARD, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
}

}  // extern "C"
