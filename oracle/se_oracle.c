/*
 * se_oracle.c -- CPU oracle of the SE fast-Gaussian-gridding path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for libse_gpu.so.  Loaded by tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py; never by the
 * product.  Each function restates the SE_fast_gridding function cited in its
 * comment (file:line of that project), keeping the floating-point operation
 * order wherever it changes the rounded result.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include "se_oracle.h"

#define ORC_PI 3.14159265358979323846

static int orc_half(int p) { return (p & 1) ? (p - 1) / 2 : p / 2; }

/* periodic index in [0,n) (SE_fgg.c:17-25 vmod) */
static int orc_pmod(int i, int n)
{
    int r = i % n;
    return r < 0 ? r + n : r;
}

static long orc_rmaj(int i, int j, int k, int n1, int n2)
{
    return ((long)i * n1 + j) * n2 + k;
}

static long orc_cmaj(int i, int j, int k, int m0, int m1)
{
    return i + (long)m0 * (j + (long)m1 * k);
}

/* ---------------------------------------------------------------- params -- */

/* SE_general.c:16-29 */
void orc_parse_params(SE_opt* opt, double xi)
{
    const double h = opt->box[0] / (double)opt->M;
    const double w = (double)opt->P * h / 2.;
    const double r = 2.0 * w * xi / opt->m;
    const double eta = r * r;
    opt->h = h;
    opt->w = w;
    opt->eta = eta;
    opt->c = 2.0 * xi * xi / eta;
    opt->xi = xi;
}

/* SE_fgg.c:69-110 (a = -1 for 3P, the z offset for 2P) */
void orc_pack_params(SE_FGG_params* p, int N, int M0, int M1, int M2, int P,
                     double c, double h, double a)
{
    memset(p, 0, sizeof(*p));
    p->N = N;
    p->P = P;
    p->P_half = orc_half(P);
    p->c = c;
    p->d = pow(c / ORC_PI, 1.5);
    p->h = h;
    p->a = a;
    p->b = -1;
    p->dims[0] = M0; p->dims[1] = M1; p->dims[2] = M2;
    p->npdims[0] = M0 + P; p->npdims[1] = M1 + P; p->npdims[2] = M2 + P;
}

/* SE_general.c:180-200 */
void orc_fcn_params(SE_FGG_params* p, const SE_opt* opt, int N)
{
    const int M = opt->M;
    orc_pack_params(p, N, M, M, M, opt->P, opt->c, opt->box[0] / M, -1.79769e+308);
    p->b = 0;
}

/* SE_general.c:517-572 (the M, m selection; the AVX build rounds M up to a
 * multiple of 4).  Returns 0; Q = sum q^2 through Q_out. */
int orc_init_params(int* M, int* P, double* m, double L, double xi,
                    const double* q, int N, double* Q_out)
{
    double Q = 0.;
    for (int i = 0; i < N; i++) Q += q[i] * q[i];
    const int Pv = *P;
    const double mm = .95 * sqrt(ORC_PI * Pv);
    const double k_inf = 2. * xi * L;
    int Ml = (int)ceil(2. * k_inf + 1) + 2;
    if (Ml < Pv) Ml = Pv;
    if (Ml % 4) Ml += 4 - Ml % 4;
    *m = mm;
    *M = Ml;
    if (Q_out) *Q_out = Q;
    return 0;
}

/* SE_fgg.c:508-535 */
void orc_base_gaussian(double* zs, const SE_FGG_params* p)
{
    const int P = p->P, ph = orc_half(P);
    const int lo = (P & 1) ? ph : ph - 1;          /* stencil is [-lo, ph] */
    const double h = p->h, c = p->c, d = p->d;
    long n = 0;
    for (int i = -lo; i <= ph; i++)
        for (int j = -lo; j <= ph; j++)
            for (int k = -lo; k <= ph; k++) {
                const double a = i * h, b = j * h, e = k * h;
                zs[n++] = d * exp(-c * (a * a + b * b + e * e));
            }
}

/* ------------------------------------------------------------- expansion -- */

/* SE_fgg.c:539-621 (3P), :625-722 (3P force), :727-819 (2P: z free, offset
 * a), :823-916 (1P: x and y free, offsets a and b, z periodic). */
int orc_expand(const double xn[3], double q, const SE_FGG_params* p, int periodicity,
               double* zx, double* zy, double* zz,
               double* zfx, double* zfy, double* zfz)
{
    const int P = p->P, ph = p->P_half;
    const double h = p->h, c = p->c;
    const int odd = P & 1;
    double t0[3];
    int first[3];
    for (int d = 0; d < 3; d++) {
        const int shifted = (periodicity == 2 && d == 2) || (periodicity == 1 && d < 2);
        const double off = (periodicity == 1 && d == 1) ? p->b : p->a;
        const double s = shifted ? off + h / 2 : 0.;
        const double u = shifted ? (xn[d] - s) / h : xn[d] / h;
        const int cell = odd ? (int)round(u) : (int)floor(u);
        first[d] = odd ? cell - ph : cell - (ph - 1);
        t0[d] = shifted ? xn[d] - (cell * h + s) : xn[d] - h * cell;
    }
    const double z3 = exp(-c * (t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2])) * q;
    double* z[3] = {zx, zy, zz};
    double* zf[3] = {zfx, zfy, zfz};
    const int lo = odd ? -ph : -ph + 1;            /* p_from of :678/:685 */
    for (int d = 0; d < 3; d++) {
        const double base = exp(2 * c * h * t0[d]);
        double v = pow(base, lo);
        z[d][0] = v;
        for (int i = 1; i < P; i++) {
            v *= base;
            z[d][i] = v;
        }
        if (zf[d])
            for (int i = 0; i < P; i++) zf[d][i] = -c * (t0[d] - (lo + i) * h);
    }
    for (int i = 0; i < P; i++) zx[i] *= z3;
    if (periodicity == 1)   /* :912-915: the free x and y corners are not shifted */
        return (int)orc_rmaj(first[0], first[1], first[2] + ph, p->npdims[1], p->npdims[2]);
    const int kz = (periodicity == 2) ? first[2] : first[2] + ph;
    return (int)orc_rmaj(first[0] + ph, first[1] + ph, kz, p->npdims[1], p->npdims[2]);
}

/* SE_fgg.c:920-963 (q = 1) */
void orc_expand_all(const SE_FGG_params* p, const double* x, int periodicity,
                    int with_force, double* zx, double* zy, double* zz,
                    double* zfx, double* zfy, double* zfz, int* idx)
{
    const int N = p->N, P = p->P;
    for (int n = 0; n < N; n++) {
        const double xn[3] = {x[n], x[n + N], x[n + 2 * N]};
        idx[n] = orc_expand(xn, 1, p, periodicity, zx + n * P, zy + n * P, zz + n * P,
                            with_force ? zfx + n * P : NULL,
                            with_force ? zfy + n * P : NULL,
                            with_force ? zfz + n * P : NULL);
    }
}

/* ---------------------------------------------------------------- spread -- */

/* SE_fgg.c:3983-4028 (force_order = 0: H += zs zz (q zx zy)) and
 * SE_fgg.c:4964-5009 (force_order = 1: H += zs zz (zx zy) q). */
void orc_grid_split(double* H, const double* q, const double* zs,
                    const double* zx, const double* zy, const double* zz,
                    const int* idx, const SE_FGG_params* p, int force_order)
{
    const int N = p->N, P = p->P, n1 = p->npdims[1], n2 = p->npdims[2];
    for (int n = 0; n < N; n++) {
        const double* ax = zx + (long)n * P;
        const double* ay = zy + (long)n * P;
        const double* az = zz + (long)n * P;
        long s = 0;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                double* row = H + idx[n] + ((long)i * n1 + j) * n2;
                if (force_order) {
                    const double cij = ax[i] * ay[j];
                    for (int k = 0; k < P; k++, s++) row[k] += zs[s] * az[k] * cij * q[n];
                } else {
                    const double cij = q[n] * ax[i] * ay[j];
                    for (int k = 0; k < P; k++, s++) row[k] += zs[s] * az[k] * cij;
                }
            }
    }
}

/* SE_fgg.c:3866-3914: the expansion is recomputed with the charge folded in */
void orc_grid(double* H, const double* x, const double* q, const double* zs,
              const SE_FGG_params* p, int periodicity)
{
    const int N = p->N, P = p->P, n1 = p->npdims[1], n2 = p->npdims[2];
    double ax[SE_P_MAX], ay[SE_P_MAX], az[SE_P_MAX];
    for (int n = 0; n < N; n++) {
        const double xn[3] = {x[n], x[n + N], x[n + 2 * N]};
        const int c0 = orc_expand(xn, q[n], p, periodicity, ax, ay, az, NULL, NULL, NULL);
        long s = 0;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                double* row = H + c0 + ((long)i * n1 + j) * n2;
                const double cij = ax[i] * ay[j];
                for (int k = 0; k < P; k++, s++) row[k] += zs[s] * az[k] * cij;
            }
    }
}

/* ----------------------------------------------------------- fold/unfold -- */

/* Elements of the periodic grid the wrap writes and the extend reads: 3P
 * M0 M1 M2, 2P M0 M1 (M2 + P); 1P the largest index its column-major map
 * i + j M0 + k M0 M1 reaches for the unfolded i < M0 + P, j < M1 + P (the
 * reference's SE1P_FGG_wrap_fcn / extend_fcn, SE_fgg.c:387-411, :478-502,
 * index H_per with the periodic strides M0, M1 over the padded x and y
 * extents, so the map overlaps itself and runs P M0 + P - 1 past M0 M1 M2). */
long orc_per_size(const SE_FGG_params* p, int periodicity)
{
    const long m0 = p->dims[0], m1 = p->dims[1], m2 = p->dims[2];
    if (periodicity == 2) return m0 * m1 * p->npdims[2];
    if (periodicity == 1) return (p->npdims[0] - 1) + (p->npdims[1] - 1) * m0 + (m2 - 1) * m0 * m1 + 1;
    return m0 * m1 * m2;
}

/* SE_fgg.c:327-352 (3P), :357-382 (2P: z is copied, not folded) and
 * :387-411 (1P: only z is folded; x and y keep their padded index).  The
 * += order is the row-major walk of H, as in the reference. */
void orc_wrap(double* H_per, const double* H, const SE_FGG_params* p, int periodicity)
{
    const int ph = orc_half(p->P);
    const int m0 = p->dims[0], m1 = p->dims[1], m2 = p->dims[2];
    const int n0 = p->npdims[0], n1 = p->npdims[1], n2 = p->npdims[2];
    long s = 0;
    if (periodicity == 1) {
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++, s++)
                    H_per[orc_cmaj(i, j, orc_pmod(k - ph, m2), m0, m1)] += H[s];
        return;
    }
    for (int i = 0; i < n0; i++) {
        const int wi = orc_pmod(i - ph, m0);
        for (int j = 0; j < n1; j++) {
            const int wj = orc_pmod(j - ph, m1);
            for (int k = 0; k < n2; k++, s++) {
                const int wk = (periodicity == 2) ? k : orc_pmod(k - ph, m2);
                H_per[orc_cmaj(wi, wj, wk, m0, m1)] += H[s];
            }
        }
    }
}

/* SE_fgg.c:417-443 (3P), :448-473 (2P) and :478-502 (1P) */
void orc_extend(double* H, const double* H_per, const SE_FGG_params* p, int periodicity)
{
    const int ph = (periodicity == 3) ? p->P_half : orc_half(p->P);
    const int m0 = p->dims[0], m1 = p->dims[1], m2 = p->dims[2];
    const int n0 = p->npdims[0], n1 = p->npdims[1], n2 = p->npdims[2];
    long s = 0;
    if (periodicity == 1) {
        for (int i = 0; i < n0; i++)
            for (int j = 0; j < n1; j++)
                for (int k = 0; k < n2; k++, s++)
                    H[s] = H_per[orc_cmaj(i, j, orc_pmod(k - ph, m2), m0, m1)];
        return;
    }
    for (int i = 0; i < n0; i++) {
        const int wi = orc_pmod(i - ph, m0);
        for (int j = 0; j < n1; j++) {
            const int wj = orc_pmod(j - ph, m1);
            for (int k = 0; k < n2; k++, s++) {
                const int wk = (periodicity == 2) ? k : orc_pmod(k - ph, m2);
                H[s] = H_per[orc_cmaj(wi, wj, wk, m0, m1)];
            }
        }
    }
}

/* ----------------------------------------------------------- interpolate -- */

/* SE_fgg.c:1176-1223; accumulate = 1 reproduces the phi[m] += of the
 * AVX unroll-4 kernel, SE_fgg.c:1856. */
void orc_int_split(double* phi, const double* H, const double* zs,
                   const double* zx, const double* zy, const double* zz,
                   const int* idx, const SE_FGG_params* p, int accumulate)
{
    const int N = p->N, P = p->P, n1 = p->npdims[1], n2 = p->npdims[2];
    const double h3 = p->h * p->h * p->h;
    for (int m = 0; m < N; m++) {
        const double* ax = zx + (long)m * P;
        const double* ay = zy + (long)m * P;
        const double* az = zz + (long)m * P;
        double acc = 0;
        long s = 0;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                const double* row = H + idx[m] + ((long)i * n1 + j) * n2;
                const double cij = ax[i] * ay[j];
                for (int k = 0; k < P; k++, s++) acc += row[k] * zs[s] * az[k] * cij;
            }
        if (accumulate) phi[m] += h3 * acc;
        else phi[m] = h3 * acc;
    }
}

/* SE_fgg.c:968-1019 */
void orc_int(double* phi, const double* H, const double* x, const double* zs,
             const SE_FGG_params* p, int periodicity)
{
    const int N = p->N, P = p->P, n1 = p->npdims[1], n2 = p->npdims[2];
    const double h3 = p->h * p->h * p->h;
    double ax[SE_P_MAX], ay[SE_P_MAX], az[SE_P_MAX];
    for (int m = 0; m < N; m++) {
        const double xm[3] = {x[m], x[m + N], x[m + 2 * N]};
        const int c0 = orc_expand(xm, 1, p, periodicity, ax, ay, az, NULL, NULL, NULL);
        double acc = 0;
        long s = 0;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                const double* row = H + c0 + ((long)i * n1 + j) * n2;
                const double cij = ax[i] * ay[j];
                for (int k = 0; k < P; k++, s++) acc += row[k] * zs[s] * az[k] * cij;
            }
        phi[m] = h3 * acc;
    }
}

/* SE_fgg.c:2241-2312 (force SoA: force[m + d N]) */
void orc_int_split_force(double* force, const double* q, const double* H,
                         const double* zs, const double* zx, const double* zy,
                         const double* zz, const double* zfx, const double* zfy,
                         const double* zfz, const int* idx, const SE_FGG_params* p)
{
    const int N = p->N, P = p->P, n1 = p->npdims[1], n2 = p->npdims[2];
    const double h3 = p->h * p->h * p->h;
    for (int m = 0; m < N; m++) {
        const long o = (long)m * P;
        double f0 = 0, f1 = 0, f2 = 0;
        long s = 0;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                const double* row = H + idx[m] + ((long)i * n1 + j) * n2;
                const double cij = zx[o + i] * zy[o + j];
                for (int k = 0; k < P; k++, s++) {
                    const double t = row[k] * zs[s] * zz[o + k] * cij * q[m];
                    f0 += t * zfx[o + i];
                    f1 += t * zfy[o + j];
                    f2 += t * zfz[o + k];
                }
            }
        force[m] = h3 * f0;
        force[m + N] = h3 * f1;
        force[m + 2 * N] = h3 * f2;
    }
}

/* SE_fgg.c:1024-1100 (the charge enters through the expansion) */
void orc_int_force(double* force, const double* H, const double* x, const double* q,
                   const double* zs, const SE_FGG_params* p)
{
    const int N = p->N, P = p->P, n1 = p->npdims[1], n2 = p->npdims[2];
    const double h3 = p->h * p->h * p->h;
    double ax[SE_P_MAX], ay[SE_P_MAX], az[SE_P_MAX];
    double fx[SE_P_MAX], fy[SE_P_MAX], fz[SE_P_MAX];
    for (int m = 0; m < N; m++) {
        const double xm[3] = {x[m], x[m + N], x[m + 2 * N]};
        const int c0 = orc_expand(xm, q[m], p, 3, ax, ay, az, fx, fy, fz);
        double f0 = 0, f1 = 0, f2 = 0;
        long s = 0;
        for (int i = 0; i < P; i++)
            for (int j = 0; j < P; j++) {
                const double* row = H + c0 + ((long)i * n1 + j) * n2;
                const double cij = ax[i] * ay[j];
                for (int k = 0; k < P; k++, s++) {
                    const double t = row[k] * zs[s] * az[k] * cij;
                    f0 += t * fx[i];
                    f1 += t * fy[j];
                    f2 += t * fz[k];
                }
            }
        force[m] = h3 * f0;
        force[m + N] = h3 * f1;
        force[m + 2 * N] = h3 * f2;
    }
}

/* --------------------------------------------------------------- k-space -- */

/* SE_general.c:34-84: FFT-ordered wave numbers 2 pi/L {0..,-..} */
void orc_k_vec(int M, const double* box, double* k1, double* k2, double* k3)
{
    double* k[3] = {k1, k2, k3};
    for (int d = 0; d < 3; d++) {
        const double f = 2.0 * ORC_PI / box[d];
        const int npos = (M % 2 == 0) ? M / 2 : (M - 1) / 2 + 1;
        for (int i = 0; i < M; i++) {
            const double j = (i < npos) ? (double)i : (double)(i - M);
            k[d][i] = f * j;
        }
    }
}

/* SE_general.c:145-175 (the non-SSE build): Z = exp(scalar k^2)/k^2 * 4 pi/M^3,
 * Z[i*n3*n2 + j*n2 + k] as indexed there. */
void orc_scaling(double scalar, double* Z, int n1, int n2, int n3, const double* box)
{
    double* k1 = malloc(sizeof(double) * n1);
    double* k2 = malloc(sizeof(double) * n1);
    double* k3 = malloc(sizeof(double) * n1);
    orc_k_vec(n1, box, k1, k2, k3);
    const double d = 4. * ORC_PI / (double)(n1 * n1 * n1);
    for (int i = 0; i < n1; i++) {
        const double ki = k1[i] * k1[i];
        for (int j = 0; j < n2; j++) {
            const double kij = ki + k2[j] * k2[j];
            const long base = (long)i * n3 * n2 + (long)j * n2;
            for (int k = 0; k < n3; k++) {
                const double K2 = kij + k3[k] * k3[k];
                Z[base + k] = exp(scalar * K2) / K2 * d;
            }
        }
    }
    free(k1); free(k2); free(k3);
}

/* SE_general.c:336-362 (complex stored as interleaved re, im) */
void orc_product_rc(double* c, const double* a, const double* b, int n, int flag)
{
    for (long i = 0; i < n; i++) {
        if (flag == -1) {
            c[2 * i] = a[2 * i] / b[i];
            c[2 * i + 1] = a[2 * i + 1] / b[i];
        } else {
            c[2 * i] = a[2 * i] * b[i];
            c[2 * i + 1] = a[2 * i + 1] * b[i];
        }
    }
}

/* ---------------------------------------------------------- direct sums -- */

/* weight of an octant term, SE_direct.c:352-371 */
static double orc_octant_weight(int a, int b, int c)
{
    const int zeros = (a == 0) + (b == 0) + (c == 0);
    return zeros == 0 ? 8. : zeros == 1 ? 4. : 2.;
}

/* SE_direct.c:377-414 */
void orc_direct_fd(double* phi, const double* x, const double* q, int N,
                   const double box[3], double xi, int layers)
{
    const double pref = 4. * ORC_PI / (box[0] * box[1] * box[2]);
#pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < N; m++) {
        double acc = 0;
        for (int a = 0; a <= layers; a++)
            for (int b = 0; b <= layers; b++)
                for (int c = 0; c <= layers; c++) {
                    if (a == 0 && b == 0 && c == 0) continue;
                    const double k0 = 2 * ORC_PI * a / box[0];
                    const double k1 = 2 * ORC_PI * b / box[1];
                    const double k2 = 2 * ORC_PI * c / box[2];
                    const double kk = k0 * k0 + k1 * k1 + k2 * k2;
                    double s = 0;
                    for (int n = 0; n < N; n++)
                        s += q[n] * cos(k0 * (x[m] - x[n])) *
                             cos(k1 * (x[m + N] - x[n + N])) *
                             cos(k2 * (x[m + 2 * N] - x[n + 2 * N]));
                    acc += orc_octant_weight(a, b, c) * s * exp(-kk / (4. * xi * xi)) / kk;
                }
        phi[m] = pref * acc;
    }
}

/* SE_direct.c:417-461 (note the factor 1/2 of :457-459) */
void orc_direct_force_fd(double* force, const double* x, const double* q, int N,
                         const double box[3], double xi, int layers)
{
    const double pref = 4. * ORC_PI / (box[0] * box[1] * box[2]);
#pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < N; m++) {
        double f[3] = {0, 0, 0};
        for (int a = -layers; a <= layers; a++)
            for (int b = -layers; b <= layers; b++)
                for (int c = -layers; c <= layers; c++) {
                    if (a == 0 && b == 0 && c == 0) continue;
                    const double k[3] = {2 * ORC_PI * a / box[0], 2 * ORC_PI * b / box[1],
                                         2 * ORC_PI * c / box[2]};
                    const double kk = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                    double s = 0;
                    for (int n = 0; n < N; n++)
                        s += q[n] * sin(k[0] * (x[n] - x[m]) + k[1] * (x[n + N] - x[m + N]) +
                                        k[2] * (x[n + 2 * N] - x[m + 2 * N]));
                    const double g = s * exp(-kk / (4. * xi * xi)) / kk;
                    for (int d = 0; d < 3; d++) f[d] += g * k[d];
                }
        for (int d = 0; d < 3; d++) force[m + d * N] = .5 * pref * f[d] * q[m];
    }
}

/* The same two sums evaluated through structure factors S(k) = sum q e^{ik.x}:
 *   phi_m   = 4pi/V sum_{k!=0} e^{-k^2/4xi^2}/k^2 Re(S(k) e^{-ik.x_m})
 *   F_{m,d} = 1/2 4pi/V q_m sum_{k!=0} e^{-k^2/4xi^2}/k^2 k_d Im(S(k) e^{-ik.x_m})
 * over the half space (k and -k contribute equally).  Targets select the
 * particles evaluated; phi/force may be NULL. */
void orc_sf_kspace(const double* x, const double* q, int N, const double box[3],
                   double xi, int jmax, double kcut2, const int* targets, int T,
                   double* phi, double* force)
{
    if (T < 0 || N <= 0 || jmax < 0) return;
    const int J = jmax + 1;
    const double pref = 4. * ORC_PI / (box[0] * box[1] * box[2]);
    /* e^{i 2pi j x_d / L_d}, j = 0..jmax, per particle and axis */
    double* tab = malloc(sizeof(double) * 2 * (size_t)J * N * 3);
    if (!tab) return;
#pragma omp parallel for
    for (int n = 0; n < N; n++)
        for (int d = 0; d < 3; d++) {
            const double th = 2 * ORC_PI * x[n + (long)d * N] / box[d];
            double* t = tab + 2 * ((size_t)(d * N + n) * J);
            for (int j = 0; j < J; j++) {
                t[2 * j] = cos(th * j);
                t[2 * j + 1] = sin(th * j);
            }
        }
    if (phi) for (int t = 0; t < T; t++) phi[t] = 0;
    if (force) for (int t = 0; t < 3 * T; t++) force[t] = 0;
    const double inv4x2 = 1. / (4. * xi * xi);
    /* parallel over (a, b) pairs of the half space a > 0, or a == 0 && b > 0,
     * or a == b == 0 && c > 0 */
    const int nab = (2 * jmax + 1) * (2 * jmax + 1);
    double* accp = phi ? calloc((size_t)T, sizeof(double)) : NULL;
    double* accf = force ? calloc((size_t)3 * T, sizeof(double)) : NULL;
#pragma omp parallel
    {
        double* lp = phi ? calloc((size_t)T, sizeof(double)) : NULL;
        double* lf = force ? calloc((size_t)3 * T, sizeof(double)) : NULL;
        double* ab = malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp for schedule(dynamic)
        for (int u = 0; u < nab; u++) {
            const int a = u / (2 * jmax + 1) - jmax;
            const int b = u % (2 * jmax + 1) - jmax;
            if (a < 0 || (a == 0 && b < 0)) continue;
            const double ka = 2 * ORC_PI * a / box[0], kb = 2 * ORC_PI * b / box[1];
            if (kcut2 > 0 && ka * ka + kb * kb > kcut2) continue;
            /* q e^{i(ka x + kb y)} */
            for (int n = 0; n < N; n++) {
                const double* ex = tab + 2 * ((size_t)(0 * N + n) * J + a);
                const double* ey = tab + 2 * ((size_t)(1 * N + n) * J + (b < 0 ? -b : b));
                const double eyr = ey[0], eyi = b < 0 ? -ey[1] : ey[1];
                ab[2 * n] = q[n] * (ex[0] * eyr - ex[1] * eyi);
                ab[2 * n + 1] = q[n] * (ex[0] * eyi + ex[1] * eyr);
            }
            const int c0 = (a == 0 && b == 0) ? 1 : -jmax;
            for (int c = c0; c <= jmax; c++) {
                const double kc = 2 * ORC_PI * c / box[2];
                const double kk = ka * ka + kb * kb + kc * kc;
                if (kcut2 > 0 && kk > kcut2) continue;
                double sr = 0, si = 0;
                for (int n = 0; n < N; n++) {
                    const double* ez = tab + 2 * ((size_t)(2 * N + n) * J + (c < 0 ? -c : c));
                    const double ezr = ez[0], ezi = c < 0 ? -ez[1] : ez[1];
                    sr += ab[2 * n] * ezr - ab[2 * n + 1] * ezi;
                    si += ab[2 * n] * ezi + ab[2 * n + 1] * ezr;
                }
                const double g = 2. * exp(-kk * inv4x2) / kk;   /* x2: the -k twin */
                for (int t = 0; t < T; t++) {
                    const int m = targets[t];
                    const double* ex = tab + 2 * ((size_t)(0 * N + m) * J + a);
                    const double* ey = tab + 2 * ((size_t)(1 * N + m) * J + (b < 0 ? -b : b));
                    const double* ez = tab + 2 * ((size_t)(2 * N + m) * J + (c < 0 ? -c : c));
                    const double eyi = b < 0 ? -ey[1] : ey[1], ezi = c < 0 ? -ez[1] : ez[1];
                    /* e^{ik.x_m} */
                    const double pr = ex[0] * ey[0] - ex[1] * eyi;
                    const double pi = ex[0] * eyi + ex[1] * ey[0];
                    const double er = pr * ez[0] - pi * ezi;
                    const double ei = pr * ezi + pi * ez[0];
                    /* S e^{-ik.x_m} */
                    const double re = sr * er + si * ei;
                    const double im = si * er - sr * ei;
                    if (lp) lp[t] += g * re;
                    if (lf) {
                        lf[3 * t] += g * im * ka;
                        lf[3 * t + 1] += g * im * kb;
                        lf[3 * t + 2] += g * im * kc;
                    }
                }
            }
        }
#pragma omp critical
        {
            if (lp) for (int t = 0; t < T; t++) accp[t] += lp[t];
            if (lf) for (int t = 0; t < 3 * T; t++) accf[t] += lf[t];
        }
        free(lp); free(lf); free(ab);
    }
    for (int t = 0; t < T; t++) {
        if (phi) phi[t] = pref * accp[t];
        if (force)
            for (int d = 0; d < 3; d++)
                force[t + d * T] = .5 * pref * accf[3 * t + d] * q[targets[t]];
    }
    free(accp); free(accf); free(tab);
}

/* ------------------------------------------------------------ reductions -- */

/* SE_fgg.c:5934-5946 */
double orc_calc_energy(const double* phi, const double* q, int N)
{
    double e = 0;
    for (int i = 0; i < N; i++) e += phi[i] * q[i];
    return e / 2.;
}

/* Stable counting sort of N keys in [0, nkeys): perm lists the input indices
 * in key order, ties in input order; offsets[nkeys+1] are the bin starts.  This
 * is the CPU statement of the binning step the GPU sort must reproduce bit for
 * bit. */
void orc_counting_sort(const int* keys, int N, int nkeys, int* perm, int* offsets)
{
    for (int b = 0; b <= nkeys; b++) offsets[b] = 0;
    for (int n = 0; n < N; n++) offsets[keys[n] + 1]++;
    for (int b = 0; b < nkeys; b++) offsets[b + 1] += offsets[b];
    int* next = malloc(sizeof(int) * (nkeys > 0 ? nkeys : 1));
    for (int b = 0; b < nkeys; b++) next[b] = offsets[b];
    for (int n = 0; n < N; n++) perm[next[keys[n]]++] = n;
    free(next);
}

/* SE_fgg.c:5894-5932: permute x (SoA) and q into ascending grid-index order.
 * The reference sorts with qsort, whose order among equal indices is
 * unspecified; this restatement keeps them in input order. */
void orc_reorder(double* x, double* q, const int* idx, int N)
{
    int lo = idx[0], hi = idx[0];
    for (int n = 1; n < N; n++) {
        if (idx[n] < lo) lo = idx[n];
        if (idx[n] > hi) hi = idx[n];
    }
    int* keys = malloc(sizeof(int) * N);
    int* perm = malloc(sizeof(int) * N);
    int* offs = malloc(sizeof(int) * (hi - lo + 2));
    for (int n = 0; n < N; n++) keys[n] = idx[n] - lo;
    orc_counting_sort(keys, N, hi - lo + 1, perm, offs);
    double* xc = malloc(sizeof(double) * 3 * N);
    double* qc = malloc(sizeof(double) * N);
    memcpy(xc, x, sizeof(double) * 3 * N);
    memcpy(qc, q, sizeof(double) * N);
    for (int i = 0; i < N; i++) {
        const int j = perm[i];
        x[i] = xc[j]; x[i + N] = xc[j + N]; x[i + 2 * N] = xc[j + 2 * N];
        q[i] = qc[j];
    }
    free(keys); free(perm); free(offs); free(xc); free(qc);
}

/* SE_direct.c:464-506 (rc > 0) and :508-549 (rc <= 0): for every target the
 * sources in index order, the images in (p0, p1, p2) nested order. */
void orc_direct_real(double* phi, const double* x, const double* q, int N,
                     const double box[3], double xi, int layers, double rc)
{
#pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < N; m++) {
        double acc = 0;
        for (int n = 0; n < N; n++) {
            const double r0 = x[m] - x[n], r1 = x[m + N] - x[n + N],
                         r2 = x[m + 2 * N] - x[n + 2 * N];
            for (int p0 = -layers; p0 <= layers; p0++)
                for (int p1 = -layers; p1 <= layers; p1++)
                    for (int p2 = -layers; p2 <= layers; p2++) {
                        if (m == n && p0 == 0 && p1 == 0 && p2 == 0) continue;
                        const double a = r0 + p0 * box[0], b = r1 + p1 * box[1],
                                     c = r2 + p2 * box[2];
                        const double r = sqrt(a * a + b * b + c * c);
                        if (rc > 0 && r > rc) continue;
                        acc += q[n] * erfc(xi * r) / r;
                    }
        }
        phi[m] += acc;
    }
}

/* SE_direct.c:551-562 */
void orc_direct_self(double* phi, const double* q, int N, double xi)
{
    const double c = 2 * xi / sqrt(ORC_PI);
    for (int m = 0; m < N; m++) phi[m] -= c * q[m];
}

/* the gradient of orc_direct_real times -q[m] (the force on m), same pairs */
void orc_direct_real_force(double* force, const double* x, const double* q, int N,
                           const double box[3], double xi, int layers, double rc)
{
    const double g = 2 * xi / sqrt(ORC_PI);
#pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < N; m++) {
        double f[3] = {0, 0, 0};
        for (int n = 0; n < N; n++) {
            const double r0 = x[m] - x[n], r1 = x[m + N] - x[n + N],
                         r2 = x[m + 2 * N] - x[n + 2 * N];
            for (int p0 = -layers; p0 <= layers; p0++)
                for (int p1 = -layers; p1 <= layers; p1++)
                    for (int p2 = -layers; p2 <= layers; p2++) {
                        if (m == n && p0 == 0 && p1 == 0 && p2 == 0) continue;
                        const double d[3] = {r0 + p0 * box[0], r1 + p1 * box[1],
                                             r2 + p2 * box[2]};
                        const double rr = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                        const double r = sqrt(rr);
                        if (rc > 0 && r > rc) continue;
                        const double s = q[n] * (erfc(xi * r) / r + g * exp(-xi * xi * rr)) / rr;
                        for (int a = 0; a < 3; a++) f[a] += s * d[a];
                    }
        }
        for (int a = 0; a < 3; a++) force[m + a * N] += q[m] * f[a];
    }
}
