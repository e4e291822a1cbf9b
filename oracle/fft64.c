/* FP64 complex FFT, arbitrary length.  See fft64.h.
 *
 * Powers of two: iterative decimation-in-time radix-2 with bit reversal.
 * Other lengths: Bluestein — x_k w_k (w_k = e^{sign i pi k^2/n}) is convolved
 * with conj(w) through a power-of-two FFT of length M >= 2n-1.
 * Twiddles are evaluated directly with cos/sin of the reduced angle so the
 * error stays at a few ulp of double for every length used in tests. */
#include "fft64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int is_pow2(size_t n) { return n && !(n & (n - 1)); }

static void fft_pow2(double *a, size_t n, int sign) {
    /* a: contiguous complex array of length n */
    size_t j = 0;
    for (size_t i = 1; i < n; i++) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = a[2 * i], ti = a[2 * i + 1];
            a[2 * i] = a[2 * j];
            a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = tr;
            a[2 * j + 1] = ti;
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        size_t half = len >> 1;
        for (size_t k = 0; k < half; k++) {
            /* angle = sign * 2 pi k / len, evaluated exactly per k */
            double ang = (double)sign * 2.0 * M_PI * (double)k / (double)len;
            double wr = cos(ang), wi = sin(ang);
            for (size_t s = 0; s < n; s += len) {
                double *u = a + 2 * (s + k), *v = a + 2 * (s + k + half);
                double vr = v[0] * wr - v[1] * wi;
                double vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr;
                v[1] = u[1] - vi;
                u[0] += vr;
                u[1] += vi;
            }
        }
    }
}

static void fft_bluestein(double *a, size_t n, int sign) {
    size_t m = 1;
    while (m < 2 * n - 1) m <<= 1;
    double *w = (double *)malloc(sizeof(double) * 2 * n);
    double *A = (double *)calloc(2 * m, sizeof(double));
    double *B = (double *)calloc(2 * m, sizeof(double));
    for (size_t k = 0; k < n; k++) {
        /* k^2 mod 2n keeps the angle small and exact */
        unsigned long long kk = ((unsigned long long)k * k) % (2ULL * n);
        double ang = (double)sign * M_PI * (double)kk / (double)n;
        w[2 * k] = cos(ang);
        w[2 * k + 1] = sin(ang);
    }
    for (size_t k = 0; k < n; k++) {
        double xr = a[2 * k], xi = a[2 * k + 1];
        A[2 * k] = xr * w[2 * k] - xi * w[2 * k + 1];
        A[2 * k + 1] = xr * w[2 * k + 1] + xi * w[2 * k];
    }
    B[0] = w[0];
    B[1] = -w[1];
    for (size_t k = 1; k < n; k++) {
        B[2 * k] = w[2 * k];
        B[2 * k + 1] = -w[2 * k + 1];
        B[2 * (m - k)] = w[2 * k];
        B[2 * (m - k) + 1] = -w[2 * k + 1];
    }
    fft_pow2(A, m, -1);
    fft_pow2(B, m, -1);
    for (size_t k = 0; k < m; k++) {
        double ar = A[2 * k], ai = A[2 * k + 1];
        double br = B[2 * k], bi = B[2 * k + 1];
        A[2 * k] = ar * br - ai * bi;
        A[2 * k + 1] = ar * bi + ai * br;
    }
    fft_pow2(A, m, +1);
    double inv = 1.0 / (double)m;
    for (size_t k = 0; k < n; k++) {
        double cr = A[2 * k] * inv, ci = A[2 * k + 1] * inv;
        a[2 * k] = cr * w[2 * k] - ci * w[2 * k + 1];
        a[2 * k + 1] = cr * w[2 * k + 1] + ci * w[2 * k];
    }
    free(w);
    free(A);
    free(B);
}

void fft64_strided(double *data, size_t n, size_t stride, int sign) {
    if (n <= 1) return;
    double *buf = data;
    if (stride != 1) {
        buf = (double *)malloc(sizeof(double) * 2 * n);
        for (size_t k = 0; k < n; k++) {
            buf[2 * k] = data[2 * k * stride];
            buf[2 * k + 1] = data[2 * k * stride + 1];
        }
    }
    if (is_pow2(n))
        fft_pow2(buf, n, sign);
    else
        fft_bluestein(buf, n, sign);
    if (stride != 1) {
        for (size_t k = 0; k < n; k++) {
            data[2 * k * stride] = buf[2 * k];
            data[2 * k * stride + 1] = buf[2 * k + 1];
        }
        free(buf);
    }
}
