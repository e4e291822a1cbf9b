/* The subset of the FFTW3 single-precision API that NewGalFinder/gsmooth.c
 * calls (gsmooth.c:45,47-51,63,97,110-112).  FFTW is not installed here, so
 * oracle/ref/fftw3_shim.c implements these entry points with an FP64 FFT
 * (float in, float out).  Test infrastructure only. */
#ifndef GF_STUB_FFTW3_H
#define GF_STUB_FFTW3_H
#include <stddef.h>
typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
#define FFTW_ESTIMATE (1U << 6)
void fftwf_plan_with_nthreads(int nthreads);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
                                 fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
                                 float *out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
#endif
