/*
 * fftw3.h -- the subset of the FFTW 3 C interface that SE_fast_gridding calls
 * (spectral_ewald.c:80,119-123,133,178-179; SE_general.c:234-270), provided by
 * libse_gpu.so on cuFFT.  FFTW itself is not used or required.
 *
 * Names, argument lists, constants and the transform conventions follow the
 * public FFTW 3 API so that the unchanged caller compiles against this header:
 *   - FFTW_FORWARD computes sum_j x_j exp(-2 pi i jk/n), FFTW_BACKWARD the same
 *     with +i; neither is normalised;
 *   - multi-dimensional arrays are row-major (last index fastest);
 *   - r2c output and c2r input hold the n0 x n1 x (n2/2+1) half spectrum.
 *
 * Plans keep raw pointers to the arrays they were made for, as FFTW plans do.
 * Host arrays are staged through device memory on every fftw_execute; managed
 * or device arrays are transformed in place on the GPU.
 */
#ifndef SE_GPU_FFTW3_SUBSET_H
#define SE_GPU_FFTW3_SUBSET_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in,
                           fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in,
                               fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in,
                               double* out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void* fftw_malloc(size_t n);
void fftw_free(void* p);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif
#endif /* SE_GPU_FFTW3_SUBSET_H */
