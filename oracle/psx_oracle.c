/*
 * psx_oracle.c -- FP64 CPU restatement of the stages of Peasoup's per-DM
 * acceleration search.  TEST INFRASTRUCTURE ONLY (see psx_oracle.h).
 *
 * Each function names the reference file:line whose behaviour it restates.
 * Build with -ffp-contract=off: the host arithmetic that the reference
 * performs in float (acceleration list, bin ranges, stretch weights) must
 * round exactly as the reference's host compiler rounds it.
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "psx_oracle.h"

/* ------------------------------------------------------------------ */
/* Resampling                                                          */
/* ------------------------------------------------------------------ */

/* src/kernels.cu:361 (device_resampleII) and :376 (device_resample):
   the product a*tsamp is a float product, the divide is in double. */
double orc_accel_fact(float acc, float tsamp)
{
    float at = acc * tsamp;
    return (double)at / (2 * 299792458.0);
}

/* Round-to-nearest-even conversion to an unsigned 64-bit index with the
   saturation of the CUDA double->ull conversion (negative -> 0). */
static uint64_t d2ull_rn(double v)
{
    if (!(v > 0.0)) return 0;
    double r = nearbyint(v); /* default rounding mode: half to even */
    if (r >= 18446744073709551615.0) return UINT64_MAX;
    return (uint64_t)r;
}

/* src/kernels.cu:321-324: index = rn(id + id*k*(id - size)), evaluated in
   double.  `fused` selects whether the final add is contracted into a
   fused multiply-add fma(id*k, id-size, id) (as an optimising CUDA
   compiler may do) or rounded after the multiply. */
void orc_resampleII_index(size_t n, float acc, float tsamp, int fused,
                          uint64_t* idx)
{
    double k = orc_accel_fact(acc, tsamp);
    double size = (double)n;
    for (size_t i = 0; i < n; ++i) {
        double id = (double)i;
        double t1 = id * k;
        double t2 = id - size;
        double v = fused ? fma(t1, t2, id) : id + t1 * t2;
        idx[i] = d2ull_rn(v);
    }
}

void orc_resampleII(const double* in, double* out, size_t n, float acc,
                    float tsamp, int fused)
{
    uint64_t* idx = (uint64_t*)malloc(sizeof(uint64_t) * n);
    orc_resampleII_index(n, acc, tsamp, fused, idx);
    for (size_t i = 0; i < n; ++i)
        out[i] = idx[i] < n ? in[idx[i]] : 0.0; /* never out of range for
                                                  physical accelerations */
    free(idx);
}

/* src/kernels.cu:315-318: centred form rn(id + k*((id-N/2)^2 - (N/2)^2)).
   fused=0: every operation rounded; fused=1: the outer add and the square
   difference contracted into fused multiply-adds. */
void orc_resample_index(size_t n, float acc, float tsamp, int fused,
                        uint64_t* idx)
{
    double k = orc_accel_fact(acc, tsamp);
    double s2 = (double)n / 2.0;
    for (size_t i = 0; i < n; ++i) {
        double id = (double)i;
        double d = id - s2;
        double q = fused ? fma(d, d, -(s2 * s2)) : d * d - s2 * s2;
        double v = fused ? fma(k, q, id) : id + k * q;
        idx[i] = d2ull_rn(v);
    }
}

/* ------------------------------------------------------------------ */
/* Spectrum forming                                                    */
/* ------------------------------------------------------------------ */

/* src/kernels.cu:216-234: amplitude |X_k|, 0 where |X_k|^2 == 0. */
void orc_form_power(const double* X, size_t nbins, double* out)
{
    for (size_t k = 0; k < nbins; ++k) {
        double re = X[2 * k], im = X[2 * k + 1];
        double z = re * re + im * im;
        out[k] = z == 0.0 ? 0.0 : sqrt(z);
    }
}

/* src/kernels.cu:238-259: sqrt(max(|X_k|^2, 0.5 |X_k - X_{k-1}|^2)) with
   X_{-1} = 0. */
void orc_form_interbin(const double* X, size_t nbins, double* out)
{
    for (size_t k = 0; k < nbins; ++k) {
        double re = X[2 * k], im = X[2 * k + 1];
        double rl = k ? X[2 * k - 2] : 0.0, il = k ? X[2 * k - 1] : 0.0;
        double a = re * re + im * im;
        double d = 0.5 * ((re - rl) * (re - rl) + (im - il) * (im - il));
        out[k] = sqrt(a > d ? a : d);
    }
}

/* ------------------------------------------------------------------ */
/* Running median (src/kernels.cu:902-1038, dereddener.hpp:41-66)      */
/* ------------------------------------------------------------------ */

static int cmp_double(const void* a, const void* b)
{
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* The median of three/five values is the middle order statistic; the
   median of four is the mean of the two middle order statistics. */
double orc_median3(double a, double b, double c)
{
    double v[3] = {a, b, c};
    qsort(v, 3, sizeof(double), cmp_double);
    return v[1];
}

double orc_median4(double a, double b, double c, double d)
{
    double v[4] = {a, b, c, d};
    qsort(v, 4, sizeof(double), cmp_double);
    return 0.5 * (v[1] + v[2]);
}

double orc_median5(double a, double b, double c, double d, double e)
{
    double v[5] = {a, b, c, d, e};
    qsort(v, 5, sizeof(double), cmp_double);
    return v[2];
}

/* src/kernels.cu:974-1008: counts 1..4 collapse to one value; otherwise
   out[i] = median of in[5i..5i+4] for i < count/5 (truncating). */
size_t orc_median_scrunch5(const double* in, size_t count, double* out)
{
    switch (count) {
    case 1: out[0] = in[0]; return 1;
    case 2: out[0] = 0.5 * (in[0] + in[1]); return 1;
    case 3: out[0] = orc_median3(in[0], in[1], in[2]); return 1;
    case 4: out[0] = orc_median4(in[0], in[1], in[2], in[3]); return 1;
    default: break;
    }
    size_t oc = count / 5;
    for (size_t i = 0; i < oc; ++i)
        out[i] = orc_median5(in[5 * i], in[5 * i + 1], in[5 * i + 2],
                             in[5 * i + 3], in[5 * i + 4]);
    return oc;
}

static size_t g_stretch_overreads = 0;
size_t orc_stretch_overreads(void) { return g_stretch_overreads; }

/* src/kernels.cu:1010-1038.  The sample position x = i*step and its
   fractional weight are float quantities in the reference (step is the
   float quotient (in_count-1)/(out_count-1), i is converted to float);
   they are reproduced in float here, the interpolation in double.  When
   float rounding puts j on the last input element with a non-zero weight
   the reference reads one element past the input; here the slope is taken
   as zero at that point and the event is counted. */
void orc_linear_stretch(const double* in, size_t in_count, double* out,
                        size_t out_count)
{
    float step = (float)(in_count - 1) / (float)(out_count - 1);
    for (size_t i = 0; i < out_count; ++i) {
        float x = (float)(unsigned)i * step;
        unsigned j = (unsigned)x;
        float w = x - (float)j;
        double v = in[j];
        if (w > 1e-5f) {
            if (j + 1 < in_count)
                v += (double)w * (in[j + 1] - in[j]);
            else
                ++g_stretch_overreads;
        }
        out[i] = v;
    }
}

/* dereddener.hpp:48-49: pos = (int)(boundary / bin_width), the float
   boundary promoted to double. */
void orc_splice_points(size_t nbins, double bin_width, float b5, float b25,
                       int* pos5, int* pos25)
{
    (void)nbins;
    *pos5 = (int)((double)b5 / bin_width);
    *pos25 = (int)((double)b25 / bin_width);
}

/* dereddener.hpp:41-62: medians of 5, 25 and 125 bins, each stretched back
   to nbins; bins below pos5 take the 5-bin curve, bins in [pos5, pos25)
   the 25-bin curve, the rest the 125-bin curve.  (The reference's second
   copy is pos25 long instead of pos25-pos5; the overrun lands in the range
   that its third copy then overwrites, so the result is the same.) */
void orc_running_median(const double* powers, size_t nbins, double bin_width,
                        float b5, float b25, double* median)
{
    size_t n5 = nbins / 5, n25 = nbins / 5 / 5, n125 = nbins / 5 / 5 / 5;
    double* m5 = (double*)malloc(sizeof(double) * (n5 + 1));
    double* m25 = (double*)malloc(sizeof(double) * (n25 + 1));
    double* m125 = (double*)malloc(sizeof(double) * (n125 + 1));
    double* tmp = (double*)malloc(sizeof(double) * nbins);
    orc_median_scrunch5(powers, nbins, m5);
    orc_median_scrunch5(m5, n5, m25);
    orc_median_scrunch5(m25, n25, m125);
    int pos5, pos25;
    orc_splice_points(nbins, bin_width, b5, b25, &pos5, &pos25);
    size_t p5 = pos5 < 0 ? 0 : (size_t)pos5;
    size_t p25 = pos25 < 0 ? 0 : (size_t)pos25;
    if (p5 > nbins) p5 = nbins;
    if (p25 > nbins) p25 = nbins;
    orc_linear_stretch(m5, n5, tmp, nbins);
    memcpy(median, tmp, sizeof(double) * p5);
    orc_linear_stretch(m25, n25, tmp, nbins);
    if (p25 > p5) memcpy(median + p5, tmp + p5, sizeof(double) * (p25 - p5));
    orc_linear_stretch(m125, n125, tmp, nbins);
    if (nbins > p25)
        memcpy(median + p25, tmp + p25, sizeof(double) * (nbins - p25));
    free(m5); free(m25); free(m125); free(tmp);
}

/* src/kernels.cu:1040-1050: X_k /= median_k; bins 0..4 are zeroed. */
void orc_deredden(double* X, const double* median, size_t nbins)
{
    for (size_t k = 0; k < nbins; ++k) {
        if (k < 5) { X[2 * k] = 0.0; X[2 * k + 1] = 0.0; continue; }
        X[2 * k] /= median[k];
        X[2 * k + 1] /= median[k];
    }
}

/* ------------------------------------------------------------------ */
/* Birdie zapping                                                      */
/* ------------------------------------------------------------------ */

static int f2i_sat(float v)
{
    if (v != v) return 0;
    if (v >= 2147483647.0f) return INT_MAX;
    if (v <= -2147483648.0f) return INT_MIN;
    return (int)v;
}

/* src/kernels.cu:1072-1082: lo = floor((f-w)/bw), hi = ceil((f+w)/bw), in
   float; lo clamped at 0, hi clamped at nbins-1; lo >= nbins -> empty. */
void orc_zap_range(float freq, float width, float bin_width, unsigned nbins,
                   int* lo, int* hi)
{
    float a = (freq - width) / bin_width;
    float b = (freq + width) / bin_width;
    int l = f2i_sat(floorf(a));
    int h = f2i_sat(ceilf(b));
    if (l < 0) l = 0;
    if (l >= (int)nbins) { *lo = 0; *hi = 0; return; }
    if (h >= (int)nbins) h = (int)nbins - 1;
    *lo = l;
    *hi = h;
}

void orc_zap(double* X, size_t nbins, float bin_width, const float* freqs,
             const float* widths, size_t nbirdies)
{
    for (size_t b = 0; b < nbirdies; ++b) {
        int lo, hi;
        orc_zap_range(freqs[b], widths[b], bin_width, (unsigned)nbins, &lo,
                      &hi);
        for (int k = lo; k < hi; ++k) { X[2 * k] = 1.0; X[2 * k + 1] = 0.0; }
    }
}

/* ------------------------------------------------------------------ */
/* Statistics                                                          */
/* ------------------------------------------------------------------ */

/* stats.hpp:25-33 with kernels.cu:433-461: rms = sqrt(sum x^2 / n),
   mean = sum x / n, std = sqrt(rms^2 - mean^2), over [first, n). */
void orc_stats(const double* x, size_t n, size_t first, double* mean,
               double* rms, double* std)
{
    double s = 0.0, s2 = 0.0;
    for (size_t i = first; i < n; ++i) { s += x[i]; s2 += x[i] * x[i]; }
    double cnt = (double)(n - first);
    *rms = sqrt(s2 / cnt);
    *mean = s / cnt;
    *std = sqrt((*rms) * (*rms) - (*mean) * (*mean));
}

/* kernels.cu:496-507: x = (x - mean) / sigma. */
void orc_normalise(double* x, size_t n, double mean, double sigma)
{
    for (size_t i = 0; i < n; ++i) x[i] = (x[i] - mean) / sigma;
}

/* kernels.cu:463-479: subtract the mean until |mean| <= 5e-7 n, at most
   102 passes.  Returns the number of passes. */
int orc_remove_baseline(double* x, size_t n)
{
    int count = 0;
    double mean;
    do {
        double s = 0.0;
        for (size_t i = 0; i < n; ++i) s += x[i];
        mean = s / (double)n;
        for (size_t i = 0; i < n; ++i) x[i] -= mean;
        if (count++ > 100) break;
    } while (fabs(mean) > 5e-7 * (double)n);
    return count;
}

/* ------------------------------------------------------------------ */
/* Harmonic sums (src/kernels.cu:34-100)                               */
/* ------------------------------------------------------------------ */

/* Fold h (1..5) adds, to the running sum that starts at in[i], the values
   in[(int)(i*m/2^h + 0.5)] for the odd m < 2^h in the reference's order
   (fold 2 adds m=3 before m=1; the other folds ascend), then stores the
   running sum times 2^(-h/2).  The index is exact integer arithmetic:
   floor((i*m + 2^(h-1)) / 2^h).  More than five folds are rejected: the
   reference's kernel fills only five. */
int orc_harmonic_sums(const double* in, size_t n, int nfolds, double* out)
{
    if (nfolds < 0 || nfolds > 5) return -1;
    static const double scale[6] = {1.0, 0.70710678118654752440, 0.5,
                                    0.35355339059327376220, 0.25,
                                    0.17677669529663688110};
    for (size_t i = 0; i < n; ++i) {
        double val = in[i];
        for (int h = 1; h <= nfolds; ++h) {
            uint64_t den = 1ull << h, half = den >> 1;
            if (h == 2) {
                val += in[(i * 3 + half) / den];
                val += in[(i * 1 + half) / den];
            } else {
                for (uint64_t m = 1; m < den; m += 2)
                    val += in[(i * m + half) / den];
            }
            out[(size_t)(h - 1) * n + i] = val * scale[h];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Peak finding (peakfinder.hpp:72-94)                                */
/* ------------------------------------------------------------------ */

/* peakfinder.hpp:78-91, with the reference's types: nyquist and factor
   are floats, orig_size an int, the power of two a double. */
void orc_peak_range(unsigned nbins, double bin_width, int nh, float min_freq,
                    float max_freq, int* start, int* end, float* factor)
{
    int size = (int)nbins;
    float nyquist = (float)(bin_width * size);
    int orig_size = (int)(2.0 * (size - 1.0));
    double p2 = pow(2.0, nh);
    int max_bin = (int)(((double)max_freq / bin_width) * p2);
    int start_idx = (int)((double)((float)orig_size * (min_freq / nyquist)) * p2);
    *start = start_idx;
    *end = size < max_bin ? size : max_bin;
    *factor = (float)(1.0 / size * (double)nyquist / pow(2.0, (double)(float)nh));
}

/* peakfinder.hpp:72-94: a cluster starts at an above-threshold bin and
   absorbs following bins while they lie closer than min_gap to the bin
   that currently holds the cluster maximum; each cluster yields its
   maximum. */
size_t orc_identify_unique_peaks(const int* idx, const double* snr,
                                 size_t count, int min_gap, int* pidx,
                                 double* psnr)
{
    size_t i = 0, np = 0;
    while (i < count) {
        double cpeak = snr[i];
        int cidx = idx[i], last = idx[i];
        ++i;
        while (i < count && (idx[i] - last) < min_gap) {
            if (snr[i] > cpeak) { cpeak = snr[i]; cidx = idx[i]; last = idx[i]; }
            ++i;
        }
        pidx[np] = cidx;
        psnr[np] = cpeak;
        ++np;
    }
    return np;
}

size_t orc_find_peaks(const double* spec, unsigned nbins, double bin_width,
                      int nh, float thresh, float min_freq, float max_freq,
                      int min_gap, int* out_idx, double* out_snr,
                      float* out_freq, size_t cap, size_t* n_above)
{
    int start, end;
    float factor;
    orc_peak_range(nbins, bin_width, nh, min_freq, max_freq, &start, &end,
                   &factor);
    if (start < 0) start = 0;
    size_t cnt = 0;
    int* ai = NULL;
    double* as = NULL;
    if (end > start) {
        ai = (int*)malloc(sizeof(int) * (size_t)(end - start));
        as = (double*)malloc(sizeof(double) * (size_t)(end - start));
        for (int i = start; i < end; ++i)
            if (spec[i] > (double)thresh) { ai[cnt] = i; as[cnt] = spec[i]; ++cnt; }
    }
    if (n_above) *n_above = cnt;
    int* pi = (int*)malloc(sizeof(int) * (cnt + 1));
    double* ps = (double*)malloc(sizeof(double) * (cnt + 1));
    size_t np = orc_identify_unique_peaks(ai, as, cnt, min_gap, pi, ps);
    size_t w = np < cap ? np : cap;
    for (size_t k = 0; k < w; ++k) {
        out_idx[k] = pi[k];
        out_snr[k] = ps[k];
        out_freq[k] = (float)pi[k] * factor;
    }
    free(ai); free(as); free(pi); free(ps);
    return np;
}

/* ------------------------------------------------------------------ */
/* Acceleration plan (include/utils/utils.hpp:143-233)                 */
/* ------------------------------------------------------------------ */

static float disp_smear(float cfreq, float ch_bw, float dm, float cdm)
{
    float ftop = (float)((double)(cfreq + ch_bw / 2) / 1e9);
    float fbot = (float)((double)(cfreq - ch_bw / 2) / 1e9);
    float ddm = fabsf(cdm - dm);
    float inv = 1.0f / (fbot * fbot) - 1.0f / (ftop * ftop);
    return (float)(4.15e-3 * (double)inv * (double)ddm);
}

static int cmp_float(const void* a, const void* b)
{
    float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

size_t orc_accel_list(float acc_lo, float acc_hi, float tol,
                      float pulse_width, size_t nsamps, float tsamp,
                      float cfreq, float ch_bw, float dm, float cdm,
                      float* out, size_t cap)
{
    ch_bw = fabsf(ch_bw);
    size_t n = 0;
    if (acc_hi == acc_lo) {
        if (cap) out[0] = acc_hi;
        return 1;
    }
#define PUSH(v) do { if (n < cap) out[n] = (v); ++n; } while (0)
    if (acc_hi >= 0 && acc_lo <= 0) PUSH(0.0f);
    float tdm = disp_smear(cfreq, ch_bw, dm, cdm);
    float sumsq = (tdm * tdm) + (pulse_width * pulse_width) + (tsamp * tsamp);
    float broad = (float)sqrt((double)sumsq);
    float factor = (float)sqrt((double)(tol * tol) - 1.0);
    float tobs = (float)nsamps * tsamp;
    float step = (float)(2.0 * (double)broad * 24.0 * 299792458.0 /
                         (double)(tobs * tobs) * (double)factor);
    float acc = acc_lo;
    while (acc <= acc_hi) {
        PUSH(acc);
        acc += step;
    }
    PUSH(acc_hi);
#undef PUSH
    if (n > cap) return n; /* caller retries with a larger buffer */
    qsort(out, n, sizeof(float), cmp_float);
    size_t u = 0;
    for (size_t i = 0; i < n; ++i)
        if (u == 0 || out[i] != out[u - 1]) out[u++] = out[i];
    return u;
}
