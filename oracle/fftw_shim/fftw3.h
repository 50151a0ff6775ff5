/*
 * Test infrastructure only: a project-written stand-in for the subset of the
 * FFTW3 API that the reference library calls.  FFTW3 itself is not installed
 * on this machine and the reference pins no version of it (its Makefile just
 * links -lfftw3f / -lfftw3).  The reference calls:
 *   fftw[f]_plan_many_dft_r2c / _c2r   (src/fk.c:256-262, src/wavelet.c:172-179,211)
 *   fftw[f]_execute, _execute_dft_r2c/_c2r (src/fk.c:326,433, src/wavelet.c:220,262,287)
 *   fftw[f]_destroy_plan, _malloc, _free, _alloc_complex
 *   fftw[f]_plan_dft_r2c_1d / _c2r_1d  (examples/make_data.c:74-77)
 * Semantics follow FFTW's published definitions: unnormalised transforms,
 * forward sign -1, r2c keeps n/2+1 bins of the last dimension, c2r treats the
 * input as the non-redundant half of a Hermitian array (imaginary parts of the
 * DC and Nyquist bins are ignored).  Only inembed/onembed == NULL with unit
 * strides is supported (the only form the reference uses).
 *
 * The arithmetic is a mixed-radix Stockham FFT written from the DFT
 * definition (fftw_shim.c).  Nothing here is derived from FFTW's source.
 */
#ifndef AGD_ORACLE_FFTW3_SHIM_H
#define AGD_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct agd_shim_plan_d *fftw_plan;
typedef struct agd_shim_plan_f *fftwf_plan;

/* double precision */
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride,
                                 int idist, fftw_complex *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out,
                               unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_execute_dft_r2c(const fftw_plan plan, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan plan, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan plan);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_complex *fftw_alloc_complex(size_t n);
double *fftw_alloc_real(size_t n);

/* single precision */
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                   float *in, const int *inembed, int istride,
                                   int idist, fftwf_complex *out,
                                   const int *onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                   fftwf_complex *in, const int *inembed,
                                   int istride, int idist, float *out,
                                   const int *onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out,
                                 unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out,
                                 unsigned flags);
void fftwf_execute(const fftwf_plan plan);
void fftwf_execute_dft_r2c(const fftwf_plan plan, float *in,
                           fftwf_complex *out);
void fftwf_execute_dft_c2r(const fftwf_plan plan, fftwf_complex *in,
                           float *out);
void fftwf_destroy_plan(fftwf_plan plan);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_complex *fftwf_alloc_complex(size_t n);
float *fftwf_alloc_real(size_t n);

#ifdef __cplusplus
}
#endif

#endif
