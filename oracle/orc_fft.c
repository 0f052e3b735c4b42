/*
 * orc_fft.c -- FP64 discrete Fourier transforms for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this file; it is
 * the checker that the parity tests and the CPU baseline run against.
 *
 * The reference performs its transforms with cuFFT (include/transforms/
 * ffter.hpp:54-110: an unnormalised forward R2C of length N and an
 * unnormalised inverse C2R of length N).  This file restates those two
 * transforms in double precision with published methods:
 *
 *   - complex transform of length 2^k: iterative radix-2 decimation in time
 *     (Cooley & Tukey 1965) with a bit-reversal permutation and twiddles
 *     evaluated directly with cos/sin of 2*pi*j/M (no recurrence, so the
 *     twiddle error stays at one rounding);
 *   - complex transform of length 3*2^k: one radix-3 Cooley-Tukey step on
 *     top of three length-2^k transforms;
 *   - real transforms of even length N through the standard half-length
 *     packing (z[j] = x[2j] + i x[2j+1], one complex transform of length
 *     N/2, then the even/odd split with twiddle exp(-+2 pi i k / N)),
 *     as described e.g. by Sorensen, Jones, Heideman & Burrus (1987).
 *
 * Sign conventions follow cuFFT: forward = exp(-2 pi i j k / N), inverse =
 * exp(+2 pi i j k / N), neither normalised.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "psx_oracle.h"

typedef double complex cplx;

static int is_pow2(size_t m) { return m && !(m & (m - 1)); }

/* In-place radix-2 DIT transform of length m (power of two). */
static void fft_pow2(cplx* a, size_t m, int sign)
{
    if (m <= 1) return;
    /* bit reversal */
    for (size_t i = 1, j = 0; i < m; ++i) {
        size_t bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { cplx t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    /* twiddle table for the largest stage: w[j] = exp(sign*2*pi*i*j/m) */
    cplx* w = (cplx*)malloc(sizeof(cplx) * (m / 2));
    const double two_pi = 6.283185307179586476925286766559;
    for (size_t j = 0; j < m / 2; ++j) {
        double ang = two_pi * (double)j / (double)m;
        w[j] = cos(ang) + sign * sin(ang) * I;
    }
    for (size_t len = 2; len <= m; len <<= 1) {
        size_t half = len >> 1, stride = m / len;
        for (size_t s = 0; s < m; s += len) {
            for (size_t k = 0; k < half; ++k) {
                cplx t = w[k * stride] * a[s + k + half];
                cplx u = a[s + k];
                a[s + k] = u + t;
                a[s + k + half] = u - t;
            }
        }
    }
    free(w);
}

/* Complex transform of length m = 2^k or 3*2^k, in place. */
static int fft_complex(cplx* a, size_t m, int sign)
{
    if (is_pow2(m)) { fft_pow2(a, m, sign); return 0; }
    if (m % 3 || !is_pow2(m / 3)) return -1;
    size_t p = m / 3;
    cplx* sub = (cplx*)malloc(sizeof(cplx) * m);
    for (size_t r = 0; r < 3; ++r) {
        for (size_t n = 0; n < p; ++n) sub[r * p + n] = a[3 * n + r];
        fft_pow2(sub + r * p, p, sign);
    }
    const double two_pi = 6.283185307179586476925286766559;
    cplx w3[3];
    for (int q = 0; q < 3; ++q) {
        double ang = two_pi * q / 3.0;
        w3[q] = cos(ang) + sign * sin(ang) * I;
    }
    for (size_t k = 0; k < p; ++k) {
        double a1 = two_pi * (double)k / (double)m;
        double a2 = two_pi * (double)(2 * k) / (double)m;
        cplx t0 = sub[k];
        cplx t1 = (cos(a1) + sign * sin(a1) * I) * sub[p + k];
        cplx t2 = (cos(a2) + sign * sin(a2) * I) * sub[2 * p + k];
        for (int q = 0; q < 3; ++q)
            a[k + q * p] = t0 + w3[q] * t1 + w3[(2 * q) % 3] * t2;
    }
    free(sub);
    return 0;
}

int orc_fft_c2c(double* data, size_t m, int sign)
{
    return fft_complex((cplx*)data, m, sign < 0 ? -1 : 1);
}

int orc_rfft(const double* in, size_t n, double* out)
{
    if (n < 2 || (n & 1)) return -1;
    size_t h = n / 2;
    cplx* z = (cplx*)malloc(sizeof(cplx) * h);
    for (size_t j = 0; j < h; ++j) z[j] = in[2 * j] + in[2 * j + 1] * I;
    if (fft_complex(z, h, -1)) { free(z); return -1; }
    cplx* X = (cplx*)out;
    const double two_pi = 6.283185307179586476925286766559;
    for (size_t k = 0; k <= h; ++k) {
        cplx zk = z[k % h];
        cplx zc = conj(z[(h - k) % h]);
        cplx e = 0.5 * (zk + zc);
        cplx o = -0.5 * I * (zk - zc);
        double ang = two_pi * (double)k / (double)n;
        X[k] = e + (cos(ang) - sin(ang) * I) * o;
    }
    free(z);
    return 0;
}

int orc_irfft(const double* in, size_t n, double* out)
{
    if (n < 2 || (n & 1)) return -1;
    size_t h = n / 2;
    const cplx* X = (const cplx*)in;
    cplx* z = (cplx*)malloc(sizeof(cplx) * h);
    const double two_pi = 6.283185307179586476925286766559;
    /* The DC and Nyquist bins of a Hermitian spectrum are real; their
       imaginary parts are discarded (as numpy's irfft does). */
    cplx x0 = creal(X[0]), xh = creal(X[h]);
    for (size_t k = 0; k < h; ++k) {
        cplx a = (k == 0) ? x0 : X[k];
        cplx b = (k == 0) ? xh : conj(X[h - k]);
        double ang = two_pi * (double)k / (double)n;
        cplx tw = cos(ang) + sin(ang) * I;
        z[k] = (a + b) + I * (a - b) * tw;
    }
    if (fft_complex(z, h, +1)) { free(z); return -1; }
    for (size_t j = 0; j < h; ++j) {
        out[2 * j] = creal(z[j]);
        out[2 * j + 1] = cimag(z[j]);
    }
    free(z);
    return 0;
}
