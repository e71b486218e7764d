// se_fftw.cu -- the FFTW 3 subset of include/fftw3.h on cuFFT.
//
// SE_fast_gridding calls FFTW for its k-space step (spectral_ewald.c:80,
// 119-123,133,178-179; SE_general.c:234-270).  Plans here wrap cuFFT plans of
// the same shape and kind; fftw_execute transforms the plan's arrays on the
// GPU (host arrays are staged through device memory, managed/device arrays
// are used in place).  fftw_malloc returns CUDA managed memory so that arrays
// allocated through it are transformed without copies.
#include <cufft.h>

#include <cstdlib>
#include <cstring>

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
    size_t in_bytes, out_bytes;
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
    if (hin || hout) {
        if (!p->din && e == cudaSuccess) e = cudaMalloc(&p->din, inplace ? big : p->in_bytes);
        if (!inplace && !p->dout && e == cudaSuccess) e = cudaMalloc(&p->dout, p->out_bytes);
    }
    if (hin) din = p->din;
    if (hout) dout = inplace ? din : p->dout;
    if (inplace && (hin != hout)) dout = din;   // mixed kinds cannot alias
    // an in-place real transform uses FFTW's (and cuFFT's) padded layout:
    // n0 x n1 x 2(n2/2 + 1) reals, the size of the half spectrum, both ways
    const size_t in_copy = inplace ? big : p->in_bytes, out_copy = inplace ? big : p->out_bytes;
    if (e == cudaSuccess && hin) e = cudaMemcpy(din, p->in, in_copy, cudaMemcpyHostToDevice);
    cufftResult r = CUFFT_SUCCESS;
    if (e == cudaSuccess) {
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
    if (e == cudaSuccess && hout) e = cudaMemcpy(p->out, dout, out_copy, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess || r != CUFFT_SUCCESS)
        fprintf(stderr, "[se_gpu] fftw_execute failed: %s / cuFFT %d\n", cudaGetErrorString(e),
                (int)r);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
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
