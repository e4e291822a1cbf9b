/* fftw3f-API shim for the reference's gsmooth.c (gsmooth.c:45-51,63,97,110-112).
 *
 * FFTW is absent from this image and its version is not pinned by the
 * reference (NewGalFinder/Makefile:20,34), so the r2c/c2r 3-D transforms are
 * evaluated here in FP64 (fft64.c) and rounded to float on output — stricter
 * than the FP32 FFTW the reference links.  Semantics follow FFTW's documented
 * contract: row-major (n0, n1, n2) real array; the in-place complex output has
 * n2/2+1 complex values per row (rows padded to 2(n2/2+1) floats); forward
 * sign -1, both directions unnormalised; c2r reads only the Hermitian half
 * (imaginary parts of the n2-direction DC and Nyquist bins are ignored).
 *
 * Test infrastructure only (oracle/_ref build).  Never linked into libgf. */
#include <stdlib.h>
#include <string.h>

#include "../fft64.h"
#include "stub/fftw3.h"

struct fftwf_plan_s {
    int n0, n1, n2;
    int r2c; /* 1: forward real-to-complex, 0: inverse complex-to-real */
    float *real;
    fftwf_complex *cplx;
};

void fftwf_plan_with_nthreads(int nthreads) { (void)nthreads; }
void *fftwf_malloc(size_t n) { return malloc(n); }
void fftwf_free(void *p) { free(p); }

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
                                 fftwf_complex *out, unsigned flags) {
    (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->n0 = n0; p->n1 = n1; p->n2 = n2; p->r2c = 1; p->real = in; p->cplx = out;
    return p;
}

fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
                                 float *out, unsigned flags) {
    (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->n0 = n0; p->n1 = n1; p->n2 = n2; p->r2c = 0; p->real = out; p->cplx = in;
    return p;
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }

/* 1-D transforms along the two outer axes of a (n0, n1, nh) complex array */
static void outer_axes(double *c, int n0, int n1, int nh, int sign) {
    for (long k = 0; k < n0; k++)
        for (long i = 0; i < nh; i++)
            fft64_strided(c + 2 * ((size_t)k * n1 * nh + i), (size_t)n1, (size_t)nh, sign);
    for (long j = 0; j < n1; j++)
        for (long i = 0; i < nh; i++)
            fft64_strided(c + 2 * ((size_t)j * nh + i), (size_t)n0, (size_t)n1 * nh, sign);
}

void fftwf_execute(const fftwf_plan p) {
    const int n0 = p->n0, n1 = p->n1, n2 = p->n2, nh = n2 / 2 + 1;
    const size_t rowf = 2 * (size_t)nh; /* padded real row length in floats */
    const size_t nrows = (size_t)n0 * n1;
    double *c = (double *)malloc(sizeof(double) * 2 * nrows * nh);
    double *row = (double *)malloc(sizeof(double) * 2 * n2);
    if (p->r2c) {
        const float *in = p->real;
        for (size_t r = 0; r < nrows; r++) {
            for (int i = 0; i < n2; i++) {
                row[2 * i] = in[r * rowf + i];
                row[2 * i + 1] = 0.0;
            }
            fft64_strided(row, (size_t)n2, 1, -1);
            memcpy(c + 2 * r * nh, row, sizeof(double) * 2 * nh);
        }
        outer_axes(c, n0, n1, nh, -1);
        float *out = (float *)p->cplx;
        for (size_t q = 0; q < 2 * nrows * nh; q++) out[q] = (float)c[q];
    } else {
        const float *in = (const float *)p->cplx;
        for (size_t q = 0; q < 2 * nrows * nh; q++) c[q] = in[q];
        outer_axes(c, n0, n1, nh, +1);
        float *out = p->real;
        for (size_t r = 0; r < nrows; r++) {
            const double *h = c + 2 * r * nh;
            for (int i = 0; i < nh; i++) {
                row[2 * i] = h[2 * i];
                row[2 * i + 1] = h[2 * i + 1];
            }
            for (int i = 1; i < n2 - i; i++) { /* Hermitian extension */
                row[2 * (n2 - i)] = h[2 * i];
                row[2 * (n2 - i) + 1] = -h[2 * i + 1];
            }
            row[1] = 0.0;                          /* DC imaginary part ignored */
            if (n2 % 2 == 0) row[2 * (n2 / 2) + 1] = 0.0; /* Nyquist likewise */
            fft64_strided(row, (size_t)n2, 1, +1);
            for (int i = 0; i < n2; i++) out[r * rowf + i] = (float)row[2 * i];
        }
    }
    free(row);
    free(c);
}
