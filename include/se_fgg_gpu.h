/*
 * se_fgg_gpu.h -- C-ABI of libse_gpu.so, the B200 implementation of the
 * Spectral Ewald fast-Gaussian-gridding (FGG) path of SE_fast_gridding.
 *
 * Part 1 (this file): the legacy entry points.  Every symbol below keeps the
 * name, the argument list and the meaning of the SE_fast_gridding function it
 * replaces (cited as file:line of that project), so that an unchanged caller
 * such as spectral_ewald.c / test_accuracy.c links against libse_gpu.so instead
 * of SE_fgg.c + SE_general.c + FFTW.  The structs are field-for-field copies of
 * SE_fgg.h:100-148 and SE_general.h:20-24, so a caller may include either this
 * header or the original ones.
 *
 * Memory: every pointer argument may be plain host memory (malloc), pinned host
 * memory, CUDA managed memory or device memory.  Host memory is staged through
 * device mirrors inside each call; managed and device memory is used in place.
 * Buffers that the library allocates (SE_FGG_allocate_*, SE_init_*_system) are
 * CUDA managed memory, so the host may read them and kernels use them without
 * copies.  Every legacy call is synchronous: when it returns, its outputs are
 * visible to the host.
 *
 * Errors: the legacy functions return void, as the originals do.  A failure
 * (CUDA error, invalid size, P > SE_P_MAX) leaves the outputs untouched, prints
 * one line to stderr and is reported by se_gpu_last_error().
 *
 * Part 2 (se_gpu.h): the device-resident API (plans, batched solves, serving).
 */
#ifndef SE_FGG_GPU_H
#define SE_FGG_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Largest Gaussian support the kernels accept (SE_fgg.h:36 P_MAX). */
#define SE_P_MAX 32

/* ---- types: layouts identical to the reference structs ------------------ */

/* SE_fgg.h:100-118 */
typedef struct
{
    double* H;      /* padded grid, (M0+P)(M1+P)(M2+P), row-major            */
    double* zs;     /* P^3 base Gaussian, row-major                          */
    double* zx;     /* N*P expansion factors (x carries exp(-c|t0|^2))        */
    double* zy;
    double* zz;
    int*    idx;    /* N linear padded indices of the stencil corners         */
    double* zfx;    /* N*P force factors -c(t0 - (p_from+i)h), FORCE only     */
    double* zfy;
    double* zfz;
    int free_zs;
    int free_fgg_expa;
} SE_FGG_work;

/* SE_fgg.h:121-134 */
typedef struct
{
    int N;
    int P;
    int P_half;
    int dims[3];
    int npdims[3];
    double c;
    double d;
    double h;
    double a;   /* z offset of the free direction (2P)                       */
    double b;
} SE_FGG_params;

/* SE_fgg.h:136-140 */
typedef struct
{
    int idx_on_grid, idx_in_array;
} idx_reorder_t;

/* SE_fgg.h:142-148 */
typedef struct
{
    double* x;      /* 3N, SoA: x[n], x[n+N], x[n+2N]                          */
    double* q;
    double* phi;
} SE_state;

/* SE_general.h:20-24 */
typedef struct
{
    double m, c, box[3], h, xi, w, eta;
    int P, M, N;
} SE_opt;

/* SE_general.h:15 */
typedef double t_complex[2];

/* ---- small helpers (SE_fgg.h:81-97; exported so -O0 callers link) -------- */
int is_odd(int p);
int isnot_div_by_4(int p);
int half(int p);

/* ---- parameters ---------------------------------------------------------- */
void SE_FGG_pack_params(SE_FGG_params*, int N, int M0, int M1, int M2,
                        int P, double c, double h);            /* SE_fgg.c:69-88   */
void SE2P_FGG_pack_params(SE_FGG_params*, int N, int M0, int M1, int M2,
                          int P, double c, double h, double a); /* SE_fgg.c:91-110  */
void SE1P_FGG_pack_params(SE_FGG_params*, int N, int M0, int M1, int M2, int P,
                          double c, double h, double a, double b); /* SE_fgg.c:113-132 */
void parse_params(SE_opt*, double xi);                        /* SE_general.c:16-29  */
void SE_FGG_FCN_params(SE_FGG_params*, const SE_opt*, int N); /* SE_general.c:180-200 */
double SE_init_params(int* M, int* P, double* m, double eps, double L,
                      double xi, const double* q, int N);     /* SE_general.c:517-572 */

/* ---- workspace (managed memory) ----------------------------------------- */
void SE_FGG_allocate_workspace(SE_FGG_work*, const SE_FGG_params*,
                               int allocate_zs, int allocate_fgg_expa);   /* SE_fgg.c:135-167 */
void SE_FGG_allocate_workspace_SSE_force(SE_FGG_work*, const SE_FGG_params*,
                                         int allocate_zs, int allocate_fgg_expa); /* SE_fgg.c:170-207 */
double* SE_FGG_allocate_grid(const SE_FGG_params*);           /* SE_fgg.c:211-217 */
double* SE_FGG_allocate_vec(int);                             /* SE_fgg.c:220-225 */
void SE_FGG_free_workspace(SE_FGG_work*);                     /* SE_fgg.c:229-243 */
void SE_FGG_free_workspace_SSE_force(SE_FGG_work*);           /* SE_fgg.c:246-263 */

/* ---- systems ------------------------------------------------------------- */
void SE_init_system(SE_state*, const SE_FGG_params*);         /* SE_fgg.c:295-312 */
void SE_init_unit_system(SE_state*, const SE_FGG_params*);    /* SE_fgg.c:266-292 */
void SE_free_system(SE_state*);                               /* SE_fgg.c:315-322 */

/* ---- utilities ----------------------------------------------------------- */
double SE_gettime(void);                                      /* SE_fgg.c:61-66 */
int SE_prod3(const int[3]);                                   /* SE_fgg.c:55-58 */
void SE_fp_set_zero(double*, int);                            /* SE_fgg.c:48-52 */
double calc_energy(SE_state, int N);                          /* SE_fgg.c:5934-5946 */
void SE_FGG_reorder_system(SE_state*, const SE_FGG_work*,
                           const SE_FGG_params*);             /* SE_fgg.c:5894-5932 */

/* ---- base Gaussian and expansion vectors ------------------------------- */
void SE_FGG_base_gaussian(SE_FGG_work*, const SE_FGG_params*);            /* SE_fgg.c:508-535 */
/* Expansion vectors with q = 1 (SE_fgg.c:920-938).  The reference picks the
 * expansion at compile time (-DTHREE_PERIODIC / -DTWO_PERIODIC /
 * -DONE_PERIODIC, SE_fgg.h:17-33); this library uses the 3P expansion
 * (SE_fgg.c:539-621) unless the process was started with SE_GPU_PERIODICITY=2
 * or 1, which selects the 2P one (SE_fgg.c:727-819) or the 1P one
 * (SE_fgg.c:823-916) for SE_FGG_expand_all, SE_FGG_grid and SE_FGG_int, as
 * those builds do. */
void SE_FGG_expand_all(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
/* FORCE factors, 3P only (the reference defines no 2P force expansion,
 * SE_fgg.h:24-27). */
void SE_FGG_expand_all_SSE_force(SE_FGG_work*, const SE_state*,
                                 const SE_FGG_params*);                   /* SE_fgg.c:941-963 */

/* 3P / 2P / 1P expansion regardless of SE_GPU_PERIODICITY (no counterpart
 * name in the reference; each equals SE_FGG_expand_all of the matching
 * build). */
void SE3P_FGG_expand_all(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE2P_FGG_expand_all(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE1P_FGG_expand_all(SE_FGG_work*, const SE_state*, const SE_FGG_params*);

/* ---- spread, POTENTIAL: H[idx+(i,j,k)] += q zx zy zz zs ----------------- */
void SE_FGG_grid(SE_FGG_work*, const SE_state*, const SE_FGG_params*);      /* SE_fgg.c:3866-3914 */
void SE_FGG_grid_split(SE_FGG_work*, const SE_state*, const SE_FGG_params*);/* SE_fgg.c:3983-4028 */
void SE_FGG_grid_split_SSE_dispatch(SE_FGG_work*, const SE_state*, const SE_FGG_params*); /* :3917-3980 */
void SE_FGG_grid_split_SSE(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_SSE_u8(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_SSE_P16(SE_FGG_work*, const SE_state*, const SE_FGG_params*);      /* :4031-4407 */
void SE_FGG_grid_split_AVX_dispatch(SE_FGG_work*, const SE_state*, const SE_FGG_params*); /* :4410-4485 */
void SE_FGG_grid_split_AVX(SE_FGG_work*, const SE_state*, const SE_FGG_params*);          /* :4488-4577 */
void SE_FGG_grid_split_AVX_P16(SE_FGG_work*, const SE_state*, const SE_FGG_params*);      /* :4580-4692 */
void SE_FGG_grid_split_AVX_P8(SE_FGG_work*, const SE_state*, const SE_FGG_params*);       /* :4695-4784 */
void SE_FGG_grid_split_AVX_u8(SE_FGG_work*, const SE_state*, const SE_FGG_params*);       /* :4786-4890 */

/* ---- spread, FORCE build (same mathematics) ----------------------------- */
void SE_FGG_grid_split_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);        /* :4964-5009 */
void SE_FGG_grid_split_SSE_dispatch_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*); /* :4895-4960 */
void SE_FGG_grid_split_SSE_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_SSE_u8_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_SSE_P16_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_AVX_dispatch_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*); /* :5392-5463 */
void SE_FGG_grid_split_AVX_P16_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_AVX_P8_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_AVX_u8_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);
void SE_FGG_grid_split_AVX_force(SE_FGG_work*, const SE_state*, const SE_FGG_params*);

/* ---- periodic fold / unfold (H_per is COLUMN-major, SE_fgg.c:326) -------- */
void SE_FGG_wrap_fcn(double* H_per, const SE_FGG_work*, const SE_FGG_params*);   /* SE_fgg.c:327-352 */
void SE2P_FGG_wrap_fcn(double* H_per, const SE_FGG_work*, const SE_FGG_params*); /* SE_fgg.c:357-382 */
void SE_FGG_extend_fcn(SE_FGG_work*, const double* H_per, const SE_FGG_params*); /* SE_fgg.c:417-443 */
void SE2P_FGG_extend_fcn(SE_FGG_work*, const double* H_per, const SE_FGG_params*); /* SE_fgg.c:448-473 */
/* 1P (z periodic, x and y free): as the reference, H_per is indexed
 * i + j M0 + k M0 M1 with the padded i < M0 + P, j < M1 + P, so it must hold
 * (M0 + P - 1) + (M1 + P - 1) M0 + (M2 - 1) M0 M1 + 1 elements (the map
 * overlaps itself; overlapping cells sum in the reference's order). */
void SE1P_FGG_wrap_fcn(double* H_per, const SE_FGG_work*, const SE_FGG_params*); /* SE_fgg.c:387-411 */
void SE1P_FGG_extend_fcn(SE_FGG_work*, const double* H_per, const SE_FGG_params*); /* SE_fgg.c:478-502 */

/* ---- interpolate, POTENTIAL: phi[m] = h^3 sum H zs zx zy zz ------------- */
void SE_FGG_int(double* phi, const SE_FGG_work*, const SE_state*, const SE_FGG_params*); /* SE_fgg.c:968-1019 */
void SE_FGG_int_split(double* phi, const SE_FGG_work*, const SE_FGG_params*);   /* SE_fgg.c:1176-1223 */
void SE_FGG_int_split_SSE_dispatch(double*, const SE_FGG_work*, const SE_FGG_params*); /* :1103-1173 */
void SE_FGG_int_split_SSE(double*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_SSE_u8(double*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_SSE_P8(double*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_SSE_P16(double*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_AVX_dispatch(double*, const SE_FGG_work*, const SE_FGG_params*); /* :1710-1764 */
/* SE_fgg.c:1768-1858 ACCUMULATES (phi[m] += ..., :1856); kept as is. */
void SE_FGG_int_split_AVX(double*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_AVX_P8(double*, const SE_FGG_work*, const SE_FGG_params*);   /* :1861-1958 */
void SE_FGG_int_split_AVX_P16(double*, const SE_FGG_work*, const SE_FGG_params*);  /* :1961-2074 */
void SE_FGG_int_split_AVX_u8(double*, const SE_FGG_work*, const SE_FGG_params*);   /* :2077-2185 */

/* ---- interpolate, FORCE: F_d[m] = h^3 q_m sum H zs zx zy zz zf_d --------- */
void SE_FGG_int_force(double* force, const SE_FGG_work*, SE_state*, const SE_FGG_params*); /* :1024-1100 */
void SE_FGG_int_split_force(double* force, SE_state*, const SE_FGG_work*, const SE_FGG_params*); /* :2241-2312 */
void SE_FGG_int_split_SSE_dispatch_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*); /* :2189-2238 */
void SE_FGG_int_split_SSE_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_SSE_P8_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_SSE_u8_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_SSE_P16_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_AVX_dispatch_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*); /* :3141-3196 */
void SE_FGG_int_split_AVX_P16_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_AVX_P8_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_AVX_u8_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);
void SE_FGG_int_split_AVX_force(double*, SE_state*, const SE_FGG_work*, const SE_FGG_params*);

/* ---- k-space (SE_general.c) ---------------------------------------------- */
void k_vec(int M, double* box, double* k1, double* k2, double* k3);        /* SE_general.c:34-84   */
void scaling(double scalar, double* Z, int n1, int n2, int n3, double* box); /* SE_general.c:145-175 */
void product_rc(t_complex* a, double* b, t_complex* c,
                int n1, int n2, int n3, int flag);                          /* SE_general.c:336-362 */
void copy_r2c(double* in, t_complex* out, int n);                          /* SE_general.c:432-440 */
void copy_c2r(t_complex* in, double* out, int n);                          /* SE_general.c:446-453 */
void do_fft_r2c_3d(double*, t_complex*, int, int, int);                    /* SE_general.c:234-240 */
void do_fft_c2r_3d(t_complex*, double*, int, int, int);                    /* SE_general.c:244-250 */
void do_fft_c2c_forward_3d(t_complex*, t_complex*, int, int, int);         /* SE_general.c:254-260 */
void do_fft_c2c_backward_3d(t_complex*, t_complex*, int, int, int);        /* SE_general.c:264-270 */
void SE_fgg_int_force(double* x, double* q, double* H, int N, SE_opt opt,
                      double* force_out);                                   /* SE_general.c:204-230 */

/* ---- library status (no counterpart in the reference) ------------------- */
/* 0 when the last legacy call on this thread succeeded, else an SE_ERR_* code. */
int se_gpu_last_error(void);
const char* se_gpu_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif /* SE_FGG_GPU_H */
