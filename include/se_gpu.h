/*
 * se_gpu.h -- device-resident API of libse_gpu.so (B200, sm_100a).
 *
 * One plan holds everything a Spectral Ewald k-space solve of one cubic,
 * three-periodic system needs on the GPU: the sorted particle records, the
 * M^3 periodic grid, the half spectrum, the cuFFT plans.  se_solve() runs the
 * path of spectral_ewald.c:20-182 (SE_fast_gridding) with no host round trip:
 *
 *   prepare -> stable counting sort by grid bin -> spread with the periodic
 *   fold fused (SE_FGG_grid + SE_FGG_wrap_fcn) -> cuFFT D2Z -> Green's
 *   function scaling (scaling/product_rc, SE_general.c:145-175,336-362) ->
 *   cuFFT Z2D -> interpolation with the periodic unfold fused (SE_FGG_extend_fcn
 *   + SE_FGG_int / SE_FGG_int_force)
 *
 * Parameters follow parse_params / SE_FGG_FCN_params (SE_general.c:16-29,
 * 180-200): h = L/M, w = P h/2, eta = (2 w xi/m)^2, c = 2 xi^2/eta,
 * d = (c/pi)^{3/2}.  Positions are SoA (x[n], x[n+N], x[n+2N]) in FP64 as in
 * the reference; FORCE output is SoA with the reference's convention
 * F = h^3 q sum H W (-c)(x - x_grid) (SE_fgg.c:1024-1100).
 *
 * Precision SE_FP64 matches the reference's FP64 CPU path to ~1e-13 relative.
 * SE_FP32 spreads and interpolates in FP32 with compensated (per-chunk FP32,
 * cross-chunk FP64) accumulation; the FFT, the scaling and the energy stay
 * FP64.
 *
 * All functions return 0 (SE_OK) or an SE_ERR_* code; pointers are device
 * pointers unless the name ends in _host; streams are cudaStream_t passed as
 * void* (NULL = the legacy default stream).  A plan may be used by one stream
 * at a time.
 */
#ifndef SE_GPU_H
#define SE_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SE_OK = 0,
    SE_ERR_CUDA = 1,
    SE_ERR_INVALID = 2,
    SE_ERR_UNSUPPORTED = 3,
    SE_ERR_NOMEM = 4,
    SE_ERR_CUFFT = 5,
    SE_ERR_INPUT = 6,    /* a position was not finite */
    SE_ERR_BUSY = 7,     /* a server's queue is full */
    SE_ERR_TIMEOUT = 8   /* a wait on a server ran out */
};

enum { SE_POTENTIAL = 0, SE_FORCE = 1 };
/* Precision of a plan or batch.  SE_FP64: every step in FP64.  SE_FP32:
 * spread and interpolation in FP32 (compensated sums), FFTs and Z(k) in FP64.
 * SE_FP32_FFT32: as SE_FP32 with the FFTs in FP32 as well (Z(k) still
 * computed in FP64 and applied to the FP32 half spectrum). */
enum { SE_FP64 = 0, SE_FP32 = 1, SE_FP32_FFT32 = 2 };

typedef struct {
    int M;              /* grid points per dimension (cubic grid)              */
    int P;              /* Gaussian support, 1 <= P <= 32                     */
    double L;           /* box side                                           */
    double xi;          /* Ewald parameter                                    */
    double m;           /* Gaussian shape factor                              */
    int mode;           /* SE_POTENTIAL or SE_FORCE                           */
    int precision;      /* SE_FP64, SE_FP32 or SE_FP32_FFT32                  */
    int max_particles;  /* capacity of the plan                               */
} se_config;

typedef struct se_plan_s* se_plan;

/* Derived FGG parameters of a configuration (no GPU needed). */
int se_config_derive(const se_config* cfg, double* h, double* w, double* eta,
                     double* c, double* d);

/* Parameters for an accuracy target (no GPU needed).  The reference's
 * SE_init_params (SE_general.c:517-572) takes P as given and prints the
 * Lindbo-Tornberg estimate of the absolute RMS error; this picks the
 * smallest P (<= 32) whose estimate is <= eps for the charges' sum of
 * squares Q in the given mode, m = 0.95 sqrt(pi P), and the reference's
 * Kolafa-Perram grid M = ceil(4 xi L + 1) + 2 (at least P), rounded up to a
 * multiple of 16 from 32 on (the tile-aligned kernels) and to even below.
 * SE_ERR_UNSUPPORTED when no P <= 32 or M <= 1024 reaches eps. */
int se_choose_params(double eps, double L, double xi, double Q, int mode, int* M, int* P,
                     double* m);
/* The estimate itself for a given P (SE_init_params' "bound for potential"
 * or "bound for force"). */
double se_error_estimate(int P, double L, double xi, double Q, int mode);

/* Device bytes a plan of this configuration holds (admission control). */
size_t se_plan_device_bytes(const se_config* cfg);

int se_plan_create(se_plan* plan, const se_config* cfg);
int se_plan_destroy(se_plan plan);

/* Kernel paths (se_plan_create_ex): which spread and interpolation kernels a
 * plan runs.  SE_PATH_TILE_SPREAD and SE_PATH_PAIR_INTERP need M a multiple
 * of 16, M >= 32 and P <= 16; SE_PATH_RUNTIME_P turns off the interpolation
 * kernels specialised for P = 8, 12, 16 (21).  SE_PATH_DEFAULT is what
 * se_plan_create does (the tile spread where it applies, the pair
 * interpolation there too from P = 8 on); SE_PATH_TUNE times
 * every valid path on the plan's configuration (synthetic uniform particles,
 * N = max_particles, at most 2^20) and keeps the fastest, remembered per
 * (M, P, mode, precision, power-of-two class of N) for the process and, with
 * the environment variable SE_GPU_TUNE_FILE set, in that file.  Every path
 * meets the same accuracy; different paths sum in different orders, so their
 * results differ in the last bits.  se_plan_device_bytes reports the default
 * path; a path mixing tile and general kernels holds 3P more factors per
 * particle. */
#define SE_PATH_DEFAULT (-1)
#define SE_PATH_TUNE (-2)
#define SE_PATH_TILE_SPREAD 1
#define SE_PATH_PAIR_INTERP 2
#define SE_PATH_RUNTIME_P 4
/* Sort the particles with the general multi-pass radix sort rather than the
 * three-kernel bin sort used where it fits (<= 8192 fine bins, <= 2^19
 * particles); both give the same permutation, so the results are identical. */
#define SE_PATH_RADIX_SORT 8
/* Run the FP64 k-space step of grids with M = 32, 64 or 128 as three
 * passes of this library's own FFT (the scaling fused into the x pass, the
 * FP32 grid copy written by the inverse pass) instead of cuFFT's D2Z, the
 * scaling pass and Z2D; the results agree to rounding (~1e-15 relative).
 * Off by default: on B200 it ties cuFFT on one M = 128 grid and is slower on
 * batches of many M = 64 grids. */
#define SE_PATH_FFT3 16
/* Stage one window per fine bin in the pair interpolation instead of one per
 * two z-adjacent bins (the FP32 default where the larger window fits three
 * CTAs per SM); both sum the same cells in the same order, so the results
 * are identical. */
#define SE_PATH_BIN_WINDOWS 32
int se_plan_create_ex(se_plan* plan, const se_config* cfg, int path);
/* The path the default choice gives a system of grid M and stencil P. */
int se_default_path(int M, int P);
/* The path a plan runs (SE_PATH_* bits). */
int se_plan_path(se_plan plan);

/* Full k-space solve on device buffers.  out: N (POTENTIAL) or 3N (FORCE).
 * phi_out (may be NULL) additionally receives the potential in FORCE mode. */
int se_solve(se_plan plan, int N, const double* x, const double* q, double* out,
             double* phi_out, void* stream);

/* The same through host buffers: copies in, solves, copies out, waits (the
 * drop-in for spectral_ewald(), which returns the result).  It runs after the
 * work already queued on `stream`, on the plan's own stream, and replays the
 * solve from a CUDA graph from its second call with the same N on (whatever
 * se_plan_set_graph says: the device buffers are the plan's own). */
int se_solve_host(se_plan plan, int N, const double* x_host, const double* q_host,
                  double* out_host, void* stream);

/* The steps, for callers that want the intermediate grid.
 * grid: M^3 FP64, row-major [x][y][z] (the transpose of the column-major
 * H_per of SE_FGG_wrap_fcn). */
int se_spread(se_plan plan, int N, const double* x, const double* q, double* grid,
              void* stream);
int se_kspace(se_plan plan, double* grid, void* stream);
int se_interp(se_plan plan, int N, const double* x, const double* q, const double* grid,
              double* out, double* phi_out, void* stream);

/* E = 1/2 sum phi q (calc_energy, SE_fgg.c:5934-5946), FP64, deterministic. */
int se_energy(const double* phi, const double* q, int N, double* energy_dev, void* stream);

/* Kernel launches the last se_solve() on this plan issued (for accounting). */
int se_plan_launch_count(se_plan plan);

/* Text of the last CUDA / cuFFT failure seen on this thread. */
const char* se_gpu_error_detail(void);

/* Per-stage timing: with timing on, each solve records CUDA events on its
 * stream; se_plan_stage_ms waits for the last solve and returns the
 * milliseconds of [prepare+sort, spread, k-space (FFT, scaling, FFT), interp]. */
int se_plan_set_timing(se_plan plan, int on);
int se_plan_stage_ms(se_plan plan, float ms[4]);

/* CUDA graphs for repeated solves (a time-stepping caller that solves the
 * same buffers again and again).  With graphs on, the first solve runs
 * directly, the second is captured into a graph and every later solve with
 * the same buffers, stream and particle count replays it; other buffers, a
 * new N or timing switched on or off capture a new graph.  System parameters
 * (L, xi, m via se_solve_system) may change between replays.  Solves on the
 * legacy default stream always run directly.  Results are identical either
 * way. */
int se_plan_set_graph(se_plan plan, int on);   /* the device-buffer entry points */

/* ------------------------------------------------- real space and self -- */
/* The other two parts of the Ewald sum, for a cubic box of edge L (device
 * buffers, accumulated into):
 *   phi[m] += sum_n sum_p q[n] erfc(xi r)/r over the images p in
 *   [-layers, layers]^3 with r = |x_m - x_n + p L|, the self image (m = n,
 *   p = 0) left out and, for rc > 0, the pairs with r > rc
 *   (SE3P_direct_real_rc, SE_direct.c:464-506; rc <= 0: SE3P_direct_real,
 *   :508-549);
 *   force[m + a N] += q[m] sum q[n] (erfc(xi r)/r + 2 xi/sqrt(pi)
 *   exp(-xi^2 r^2)) r_a / r^2 over the same pairs: the force of that
 *   potential (the reference has no real-space force).
 * phi or force may be NULL (not both).  Cutoffs 0 < rc <= L/2 with at least
 * three cells of edge >= rc per axis use a cell list (positions anywhere
 * within +-511 boxes; scratch from the stream-ordered pool); the others all
 * pairs, in the reference's order of summation. */
int se_real_space(const double* x, const double* q, int N, double L, double xi, int layers,
                  double rc, double* phi, double* force, void* stream);
/* phi[m] -= 2 xi / sqrt(pi) q[m]: SE3P_direct_self (SE_direct.c:551-562). */
int se_self_term(const double* q, int N, double xi, double* phi, void* stream);

/* FP32 FMA throughput (TFLOP/s) of the current GPU from an FMA-chain kernel:
 * the compute roofline of the spread and interpolation kernels. */
int se_probe_fma_tflops(double* tflops, void* stream);

/* Stable counting sort of N keys in [0, nkeys): perm[s] = input index of the
 * s-th smallest key, ties in input order; offsets[nkeys+1] bin starts.
 * Device buffers; scratch from se_sort_scratch_bytes(). */
size_t se_sort_scratch_bytes(int N, int nkeys);
int se_counting_sort(const int* keys, int N, int nkeys, int* perm, int* offsets,
                     void* scratch, size_t scratch_bytes, void* stream);

/* The same sort for callers that cannot allocate device memory when they
 * sort (a frozen or captured memory pool, host callbacks, real-time loops, a
 * library that does not own the process's allocator).  No counterpart in the
 * reference.  It allocates nothing: its working memory is a device array of
 * SE_SORT_STATIC_BYTES inside the library (held on every GPU that loads the
 * library, until exit), so N <= SE_SORT_STATIC_MAX_N and
 * nkeys <= SE_SORT_STATIC_MAX_KEYS; larger sizes return SE_ERR_INVALID.
 * The first call on a device resolves the array's address and should come
 * before any stream capture; the address is kept for the life of the
 * process, which assumes the device's primary context is never reset
 * (no cudaDeviceReset between calls).  Calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller.  Results are identical
 * to se_counting_sort. */
#define SE_SORT_STATIC_MAX_N 262144
#define SE_SORT_STATIC_MAX_KEYS 65536
#define SE_SORT_STATIC_BYTES (6u << 20)
int se_counting_sort_static(const int* keys, int N, int nkeys, int* perm, int* offsets,
                            void* stream);

/* ---------------------------------------------------------------- batch -- */
/* Many independent systems solved together: one sort, one spread launch and
 * one interpolation launch over all systems through per-system offset
 * tables, and one batched cuFFT plan per distinct grid size. */
typedef struct {
    int N;
    int M;
    int P;
    double L;
    double xi;
    double m;
    int mode;           /* SE_POTENTIAL or SE_FORCE */
} se_system;

typedef struct se_batch_s* se_batch;

int se_batch_create(se_batch* batch, const se_system* systems, int nsys, int precision);
/* The same with each system's kernel path (SE_PATH_* bits; NULL: the
 * defaults, as se_batch_create). */
int se_batch_create_ex(se_batch* batch, const se_system* systems, int nsys, int precision,
                       const int* paths);
int se_batch_destroy(se_batch batch);
size_t se_batch_device_bytes(const se_system* systems, int nsys, int precision);
/* x: concatenated per-system SoA blocks (3 N_s each), q: concatenated N_s,
 * out: concatenated N_s (POTENTIAL) or 3 N_s (FORCE) blocks. */
int se_batch_solve(se_batch batch, const double* x, const double* q, double* out,
                   void* stream);
int se_batch_launch_count(se_batch batch);
int se_batch_set_timing(se_batch batch, int on);
int se_batch_stage_ms(se_batch batch, float ms[4]);
/* The same CUDA-graph replay as se_plan_set_graph, for a batch. */
int se_batch_set_graph(se_batch batch, int on);

/* Solve one system on a plan made for the same M, P and mode, with the
 * system's own N (<= the plan's max_particles), L, xi and m.  The plan's
 * device table is rewritten in stream order, so a plan kept per (M, P, mode)
 * serves systems of any box size and particle count without a host wait.
 * Results are identical to a plan created for exactly this system. */
int se_solve_system(se_plan plan, const se_system* sys, const double* x, const double* q,
                    double* out, double* phi_out, void* stream);

/* -------------------------------------------------------------- serving -- */
/* A request loop on the current GPU (no counterpart in the reference).
 * Requests are queued as they arrive and admitted first come, first served
 * whenever a solve slot (a CUDA stream) is free and the plan the request
 * needs fits the device-memory budget.  Plans (grid, spectrum, particle and
 * staging buffers, cuFFT plans) are cached by (M, P, mode, capacity class) and
 * stay resident between requests; an idle plan is freed, least recently used
 * first, only when a new one would not otherwise fit.  Admitted solves run on
 * their own streams and overlap on the device, so requests that arrive while
 * others are running start as soon as a slot and memory are free.  Each
 * result is bit-identical to se_solve_system on the same inputs, alone or in
 * any mix.  Host requests should use pinned memory: a copy from or to
 * pageable memory makes the loop wait for it. */
#define SE_WHERE_HOST 0     /* x, q, out are host memory */
#define SE_WHERE_DEVICE 1   /* x, q, out are device memory on the server's GPU */

typedef struct {
    int slots;          /* solves in flight at once, 1..64                     */
    int precision;      /* SE_FP32, SE_FP32_FFT32 or SE_FP64                   */
    size_t hbm_budget;  /* device bytes the server may hold (plans + staging)  */
    int max_queue;      /* queued requests before submit says SE_ERR_BUSY; 0: no limit */
} se_server_config;

typedef struct {
    se_system sys;      /* N, M, P, L, xi, m, mode                             */
    const double* x;    /* 3N positions, SoA; valid until the request completes */
    const double* q;    /* N charges                                           */
    double* out;        /* N potentials (POTENTIAL) or 3N forces, SoA (FORCE)  */
    int where;          /* SE_WHERE_HOST or SE_WHERE_DEVICE                    */
} se_request;

typedef struct {
    long long ticket;
    int status;         /* SE_OK, SE_ERR_INPUT (a position was not finite), ... */
    double queue_s;     /* submit to admission                                 */
    double latency_s;   /* submit to result in place                           */
} se_completion;

typedef struct {
    long long submitted, completed, failed;
    int queued, in_flight, plans;
    long long plans_created, plans_evicted;
    size_t hbm_used, hbm_peak;
} se_server_stats;

typedef struct se_server_s* se_server;

/* Device bytes the server charges for a request's plan (admission unit). */
size_t se_server_request_bytes(const se_system* sys, int precision);
int se_server_create(se_server* server, const se_server_config* cfg);
/* Builds and caches plans for these systems now (a warm cache). */
int se_server_reserve(se_server server, const se_system* systems, int n);
/* Queues a request; SE_ERR_NOMEM if its plan alone exceeds the budget. */
int se_server_submit(se_server server, const se_request* req, long long* ticket);
/* Moves up to max completions (in completion order) into done, no waiting. */
int se_server_poll(se_server server, se_completion* done, int max, int* n_done);
/* Waits until every submitted request has completed (SE_ERR_TIMEOUT after
 * timeout_s seconds; a negative timeout waits without limit). */
int se_server_drain(se_server server, double timeout_s);
int se_server_get_stats(se_server server, se_server_stats* stats);
/* Drains, then frees every plan, stream and buffer. */
int se_server_destroy(se_server server);

#ifdef __cplusplus
}
#endif
#endif /* SE_GPU_H */
