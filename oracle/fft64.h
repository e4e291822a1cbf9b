/* FP64 complex FFT of arbitrary length (iterative radix-2 for powers of two,
 * Bluestein's chirp-z algorithm for every other length).
 *
 * Test infrastructure only: it backs the fftw3f-API shim that lets the
 * reference's gsmooth.c run without FFTW, and the oracle's spectral checks.
 * It is never linked into the product library. */
#ifndef GF_ORACLE_FFT64_H
#define GF_ORACLE_FFT64_H
#include <stddef.h>

/* In-place transform of n interleaved (re, im) doubles separated by `stride`
 * complex elements.  sign = -1 is the forward transform e^{-2 pi i jk/n},
 * sign = +1 the unnormalised inverse (FFTW's sign convention). */
void fft64_strided(double *data, size_t n, size_t stride, int sign);

#endif
