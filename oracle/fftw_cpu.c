/*
 * fftw_cpu.c -- a CPU provider of the FFTW 3 subset in include/fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY.  FFTW is not installed in this image, so the
 * reference (whose spectral_ewald.c / SE_general.c call fftw_plan_dft_3d,
 * fftw_execute and fftw_destroy_plan) is linked against this file to run on
 * the CPU as the oracle and as the timed CPU baseline.  It is a plain
 * mixed-radix Cooley-Tukey FFT written for this project (radix 2, 3, 4, 5
 * butterflies, a direct DFT for other prime factors), applied axis by axis.
 * Conventions are FFTW's: FORWARD uses exp(-2 pi i jk/n), no normalisation,
 * row-major arrays, r2c / c2r on the n0 x n1 x (n2/2+1) half spectrum.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "fftw3.h"

/* Wall time spent inside fftw_execute since the last fc_fft_reset(): the CPU
 * baseline reports the FFT's share of a reference solve with it. */
static double fc_fft_time;

double fc_fft_seconds(void) { return fc_fft_time; }
void fc_fft_reset(void) { fc_fft_time = 0; }

static double fc_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

#define FC_PI 3.14159265358979323846

typedef struct { double re, im; } fc_cplx;

enum { FC_C2C, FC_R2C, FC_C2R };

struct fftw_plan_s {
    int n[3];
    int kind;
    int sign;
    void* in;
    void* out;
};

/* ---------------------------------------------------------- 1-D FFT -- */

static int fc_smallest_factor(int n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int f = 3; f * f <= n; f += 2)
        if (n % f == 0) return f;
    return n;
}

/* out[k] = sum_j in[j*stride] w^(jk), n points; w = exp(sign 2 pi i / n)
 * tw holds exp(sign 2 pi i t / ntot) for t < ntot, with n | ntot. */
static void fc_fft_rec(const fc_cplx* in, long stride, fc_cplx* out, int n,
                       const fc_cplx* tw, int ntot, fc_cplx* scratch)
{
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int r = fc_smallest_factor(n);
    const int m = n / r;
    /* sub-transforms of the r decimated sequences, into out[s*m ..] */
    for (int s = 0; s < r; s++)
        fc_fft_rec(in + s * stride, stride * r, out + s * m, m, tw, ntot, scratch);
    const int step = ntot / n;   /* tw index of w_n^1 */
    for (int k = 0; k < m; k++) {
        fc_cplx v[64];
        fc_cplx* t = (r <= 64) ? v : scratch;
        for (int s = 0; s < r; s++) {
            /* twiddle w_n^{s k} */
            const fc_cplx a = out[s * m + k];
            const long e = ((long)s * k * step) % ntot;
            const fc_cplx w = tw[e];
            t[s].re = a.re * w.re - a.im * w.im;
            t[s].im = a.re * w.im + a.im * w.re;
        }
        if (r == 2) {
            out[k].re = t[0].re + t[1].re; out[k].im = t[0].im + t[1].im;
            out[k + m].re = t[0].re - t[1].re; out[k + m].im = t[0].im - t[1].im;
        } else if (r == 4) {
            /* w_4 = tw[ntot/4] = +-i */
            const double sg = tw[ntot / 4].im;   /* +1 or -1 */
            const fc_cplx a0 = {t[0].re + t[2].re, t[0].im + t[2].im};
            const fc_cplx a1 = {t[0].re - t[2].re, t[0].im - t[2].im};
            const fc_cplx b0 = {t[1].re + t[3].re, t[1].im + t[3].im};
            const fc_cplx b1 = {t[1].re - t[3].re, t[1].im - t[3].im};
            /* i*sg*b1 */
            const fc_cplx jb1 = {-sg * b1.im, sg * b1.re};
            out[k].re = a0.re + b0.re; out[k].im = a0.im + b0.im;
            out[k + m].re = a1.re + jb1.re; out[k + m].im = a1.im + jb1.im;
            out[k + 2 * m].re = a0.re - b0.re; out[k + 2 * m].im = a0.im - b0.im;
            out[k + 3 * m].re = a1.re - jb1.re; out[k + 3 * m].im = a1.im - jb1.im;
        } else {
            /* direct r-point DFT with w_r = tw[ntot/r] */
            const int rs = ntot / r;
            for (int q = 0; q < r; q++) {
                double sr = 0, si = 0;
                for (int s = 0; s < r; s++) {
                    const fc_cplx w = tw[((long)s * q % r) * rs];
                    sr += t[s].re * w.re - t[s].im * w.im;
                    si += t[s].re * w.im + t[s].im * w.re;
                }
                out[k + q * m].re = sr;
                out[k + q * m].im = si;
            }
        }
    }
}

/* in-place transform of one line of n points at stride (in elements) */
static void fc_fft_line(fc_cplx* data, long stride, int n, int sign,
                        const fc_cplx* tw, fc_cplx* buf, fc_cplx* tmp, fc_cplx* scratch)
{
    for (int j = 0; j < n; j++) buf[j] = data[j * stride];
    fc_fft_rec(buf, 1, tmp, n, tw, n, scratch);
    for (int j = 0; j < n; j++) data[j * stride] = tmp[j];
    (void)sign;
}

static fc_cplx* fc_twiddles(int n, int sign)
{
    fc_cplx* tw = malloc(sizeof(fc_cplx) * n);
    for (int t = 0; t < n; t++) {
        const double a = sign * 2.0 * FC_PI * (double)t / (double)n;
        tw[t].re = cos(a);
        tw[t].im = sin(a);
    }
    return tw;
}

/* 3-D complex transform, in place, row-major n0 x n1 x n2 */
static void fc_fft3(fc_cplx* a, const int n[3], int sign)
{
    const long s[3] = {(long)n[1] * n[2], n[2], 1};
    for (int axis = 2; axis >= 0; axis--) {
        const int len = n[axis];
        if (len <= 1) continue;
        fc_cplx* tw = fc_twiddles(len, sign);
        const long total = (long)n[0] * n[1] * n[2];
        const long lines = total / len;
#pragma omp parallel
        {
            fc_cplx* buf = malloc(sizeof(fc_cplx) * len);
            fc_cplx* tmp = malloc(sizeof(fc_cplx) * len);
            fc_cplx* scr = malloc(sizeof(fc_cplx) * len);
#pragma omp for
            for (long l = 0; l < lines; l++) {
                /* base offset of line l: enumerate the two other axes */
                long base;
                if (axis == 2) base = l * n[2];
                else if (axis == 1) base = (l / n[2]) * s[0] + (l % n[2]);
                else base = l;
                fc_fft_line(a + base, s[axis], len, sign, tw, buf, tmp, scr);
            }
            free(buf); free(tmp); free(scr);
        }
        free(tw);
    }
}

/* ------------------------------------------------------------ API -- */

static fftw_plan fc_new(int n0, int n1, int n2, int kind, int sign, void* in, void* out)
{
    fftw_plan p = malloc(sizeof(*p));
    p->n[0] = n0; p->n[1] = n1; p->n[2] = n2;
    p->kind = kind; p->sign = sign; p->in = in; p->out = out;
    return p;
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in,
                           fftw_complex* out, int sign, unsigned flags)
{
    (void)flags;
    return fc_new(n0, n1, n2, FC_C2C, sign, in, out);
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in,
                               fftw_complex* out, unsigned flags)
{
    (void)flags;
    return fc_new(n0, n1, n2, FC_R2C, FFTW_FORWARD, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in,
                               double* out, unsigned flags)
{
    (void)flags;
    return fc_new(n0, n1, n2, FC_C2R, FFTW_BACKWARD, in, out);
}

static void fc_execute(const fftw_plan p);

void fftw_execute(const fftw_plan p)
{
    const double t0 = fc_now();
    fc_execute(p);
    fc_fft_time += fc_now() - t0;
}

static void fc_execute(const fftw_plan p)
{
    const long tot = (long)p->n[0] * p->n[1] * p->n[2];
    const int nh = p->n[2] / 2 + 1;
    if (p->kind == FC_C2C) {
        if (p->out != p->in) memcpy(p->out, p->in, sizeof(fc_cplx) * tot);
        fc_fft3((fc_cplx*)p->out, p->n, p->sign);
    } else if (p->kind == FC_R2C) {
        fc_cplx* a = malloc(sizeof(fc_cplx) * tot);
        const double* r = (const double*)p->in;
        for (long i = 0; i < tot; i++) { a[i].re = r[i]; a[i].im = 0; }
        fc_fft3(a, p->n, FFTW_FORWARD);
        fc_cplx* o = (fc_cplx*)p->out;
        for (long ij = 0; ij < (long)p->n[0] * p->n[1]; ij++)
            for (int k = 0; k < nh; k++) o[ij * nh + k] = a[ij * p->n[2] + k];
        free(a);
    } else {
        fc_cplx* a = malloc(sizeof(fc_cplx) * tot);
        const fc_cplx* h = (const fc_cplx*)p->in;
        const int n0 = p->n[0], n1 = p->n[1], n2 = p->n[2];
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++) {
                    fc_cplx v;
                    if (k < nh) {
                        v = h[((long)i * n1 + j) * nh + k];
                    } else {   /* Hermitian twin */
                        const int ii = (n0 - i) % n0, jj = (n1 - j) % n1, kk = n2 - k;
                        v = h[((long)ii * n1 + jj) * nh + kk];
                        v.im = -v.im;
                    }
                    a[((long)i * n1 + j) * n2 + k] = v;
                }
        fc_fft3(a, p->n, FFTW_BACKWARD);
        double* r = (double*)p->out;
        for (long i = 0; i < tot; i++) r[i] = a[i].re;
        free(a);
    }
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
void* fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void* p) { free(p); }
void fftw_cleanup(void) {}
