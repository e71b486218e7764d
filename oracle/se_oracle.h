/*
 * se_oracle.h -- CPU oracle of the SE fast-Gaussian-gridding path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load this library, and only as the checker.  The
 * product (libse_gpu.so) never links or calls it.
 *
 * Every function restates the algorithm of SE_fast_gridding at the cited
 * file:line, in the same floating-point operation order where that order is
 * observable, so that the oracle agrees with the reference to the last bit on
 * the golden vectors in tests/golden/ (generated from the reference compiled
 * from source, see oracle/Makefile and tests/golden/make_golden.py).
 */
#ifndef SE_ORACLE_H
#define SE_ORACLE_H

#include "se_fgg_gpu.h"   /* SE_FGG_params / SE_opt layouts */

#ifdef __cplusplus
extern "C" {
#endif

/* parameters */
void orc_parse_params(SE_opt* opt, double xi);
void orc_fcn_params(SE_FGG_params* p, const SE_opt* opt, int N);
void orc_pack_params(SE_FGG_params* p, int N, int M0, int M1, int M2, int P,
                     double c, double h, double a);
int  orc_init_params(int* M, int* P, double* m, double L, double xi,
                     const double* q, int N, double* Q_out);

/* base Gaussian zs[P^3] */
void orc_base_gaussian(double* zs, const SE_FGG_params* p);

/* expansion of one particle; periodicity 3, 2 or 1; zf* may be NULL */
int orc_expand(const double xn[3], double q, const SE_FGG_params* p, int periodicity,
               double* zx, double* zy, double* zz,
               double* zfx, double* zfy, double* zfz);
void orc_expand_all(const SE_FGG_params* p, const double* x, int periodicity,
                    int with_force, double* zx, double* zy, double* zz,
                    double* zfx, double* zfy, double* zfz, int* idx);

/* spread */
void orc_grid_split(double* H, const double* q, const double* zs,
                    const double* zx, const double* zy, const double* zz,
                    const int* idx, const SE_FGG_params* p, int force_order);
void orc_grid(double* H, const double* x, const double* q, const double* zs,
              const SE_FGG_params* p, int periodicity);

/* fold / unfold; H_per column-major */
long orc_per_size(const SE_FGG_params* p, int periodicity);
void orc_wrap(double* H_per, const double* H, const SE_FGG_params* p, int periodicity);
void orc_extend(double* H, const double* H_per, const SE_FGG_params* p, int periodicity);

/* interpolate */
void orc_int_split(double* phi, const double* H, const double* zs,
                   const double* zx, const double* zy, const double* zz,
                   const int* idx, const SE_FGG_params* p, int accumulate);
void orc_int(double* phi, const double* H, const double* x, const double* zs,
             const SE_FGG_params* p, int periodicity);
void orc_int_split_force(double* force, const double* q, const double* H,
                         const double* zs, const double* zx, const double* zy,
                         const double* zz, const double* zfx, const double* zfy,
                         const double* zfz, const int* idx, const SE_FGG_params* p);
void orc_int_force(double* force, const double* H, const double* x, const double* q,
                   const double* zs, const SE_FGG_params* p);

/* k-space */
void orc_k_vec(int M, const double* box, double* k1, double* k2, double* k3);
void orc_scaling(double scalar, double* Z, int n1, int n2, int n3, const double* box);
void orc_product_rc(double* c, const double* a, const double* b, int n, int flag);

/* direct Fourier-space Ewald sums (O(N^2 layers^3), cube |j|<=layers) */
void orc_direct_fd(double* phi, const double* x, const double* q, int N,
                   const double box[3], double xi, int layers);
void orc_direct_force_fd(double* force, const double* x, const double* q, int N,
                         const double box[3], double xi, int layers);
/* real-space Ewald sums over the periodic images p in [-layers, layers]^3:
 * phi[m] += sum_n sum_p q[n] erfc(xi r) / r, r = |x_m - x_n + p box|, the
 * self image (m = n, p = 0) left out, pairs with r > rc left out when rc > 0
 * (SE3P_direct_real_rc / SE3P_direct_real); self term phi[m] -= 2 xi/sqrt(pi)
 * q[m] (SE3P_direct_self); the real-space force, the gradient of the same
 * sum (no counterpart in the reference): force[m + aN] += q[m] sum q[n]
 * (erfc(xi r)/r + 2 xi/sqrt(pi) exp(-xi^2 r^2)) r_a / r^2 */
void orc_direct_real(double* phi, const double* x, const double* q, int N,
                     const double box[3], double xi, int layers, double rc);
void orc_direct_self(double* phi, const double* q, int N, double xi);
void orc_direct_real_force(double* force, const double* x, const double* q, int N,
                           const double box[3], double xi, int layers, double rc);
/* the same sums through structure factors, O(K N); jmax: cube half-width,
 * kcut2 > 0 restricts to |k|^2 <= kcut2 (a converged sphere) */
void orc_sf_kspace(const double* x, const double* q, int N, const double box[3],
                   double xi, int jmax, double kcut2, const int* targets, int T,
                   double* phi, double* force);

/* reductions, sorting */
double orc_calc_energy(const double* phi, const double* q, int N);
void orc_counting_sort(const int* keys, int N, int nkeys, int* perm, int* offsets);
void orc_reorder(double* x, double* q, const int* idx, int N);

#ifdef __cplusplus
}
#endif
#endif
