// psx_device.cuh -- per-element arithmetic of the search stages.  Every
// kernel of the library (the single-stage drop-in entry points and the
// fused search kernels) calls these, so that all paths round identically.
// Expressions that must round as the reference's do are written in the
// same operation order as the cited reference lines.
#pragma once
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace psx {

// ---- resampling (reference src/kernels.cu:315-324) --------------------
// Read index of output sample i for the "II" resampler: the quadratic
// time-shift i*k*(i-N) added to i in double precision, rounded to the
// nearest integer (ties to even).
__device__ __forceinline__ unsigned long long resampleII_index(
    unsigned long long i, double k, double size)
{
    return __double2ull_rn(i + i * k * (i - size));
}

// Sample at a resample read index.  For physical accelerations the index
// stays inside [0, N) (|k| N < 1/2 would be needed to leave it, i.e.
// |a| ~ c/(N tsamp), 10^5 m/s^2 and more); beyond that the series is taken
// as zero instead of reading outside the buffer as the reference would.
__device__ __forceinline__ float gather_at(const float* __restrict__ in,
                                           unsigned long long idx,
                                           unsigned long long n)
{
    return idx < n ? in[idx] : 0.0f;
}

// resampleII read with the output index i given as an exact double and
// n < 2^32: the expression of resampleII_index, rounded by the same mode to
// a 32-bit index (both conversions clamp, so indices outside [0, n) read
// zero in both forms).  The resample kernel and the gather of the two-pass
// transform both read through this.
__device__ __forceinline__ float resampleII_read(const float* __restrict__ in, double i, double k,
                                                 double size, unsigned n)
{
    const unsigned idx = __double2uint_rn(i + i * k * (i - size));
    return idx < n ? in[idx] : 0.0f;
}

// Read index of the centred resampler: k*((i-N/2)^2 - (N/2)^2).
__device__ __forceinline__ unsigned long long resample_index(
    unsigned long long i, double k, double size_by_2)
{
    return __double2ull_rn(i + k * (((i - size_by_2) * (i - size_by_2)) -
                                    (size_by_2 * size_by_2)));
}

// ---- spectrum forming (reference src/kernels.cu:216-259) --------------
__device__ __forceinline__ float amplitude(float re, float im)
{
    float z = re * re + im * im;
    return z == 0 ? 0.0f : z * rsqrtf(z);
}

// Interbinned amplitude of bin k given bin k-1 (zero for k == 0).
__device__ __forceinline__ float interbin(float re, float im, float re_l,
                                          float im_l)
{
    float ampsq = re * re + im * im;
    float ampsq_diff = 0.5f * ((re - re_l) * (re - re_l) +
                               (im - im_l) * (im - im_l));
    return sqrtf(fmaxf(ampsq, ampsq_diff));
}

// Normalisation (reference src/kernels.cu:503-506): subtract, then divide.
__device__ __forceinline__ float normalise(float v, float mean, float sigma)
{
    v -= mean;
    v /= sigma;
    return v;
}

// ---- medians (the order statistics of reference src/kernels.cu:902-956)
// Median of five: order the pairs (a,b) and (c,d); the smaller of a and c
// is below three of the four and cannot be the median, so replace its
// pair's low element with e and re-order that pair; the median is then
// the second smallest of the two ordered pairs.
__device__ __forceinline__ float med5(float a, float b, float c, float d,
                                      float e)
{
    float t;
    if (b < a) { t = a; a = b; b = t; }
    if (d < c) { t = c; c = d; d = t; }
    if (a < c) {
        a = e;
        if (b < a) { t = a; a = b; b = t; }
    } else {
        c = e;
        if (d < c) { t = c; c = d; d = t; }
    }
    return fminf(fmaxf(a, c), fminf(b, d));
}

__device__ __forceinline__ float med3(float a, float b, float c)
{
    return fmaxf(fminf(a, b), fminf(fmaxf(a, b), c));
}

// Mean of the two middle order statistics of four values.
__device__ __forceinline__ float med4(float a, float b, float c, float d)
{
    float lo1 = fminf(a, b), hi1 = fmaxf(a, b);
    float lo2 = fminf(c, d), hi2 = fmaxf(c, d);
    return 0.5f * (fmaxf(lo1, lo2) + fminf(hi1, hi2));
}

// ---- linear stretch (reference src/kernels.cu:1010-1023) --------------
// Value at output sample i of `in` (in_count samples) stretched with the
// float step (in_count-1)/(out_count-1).  The sample position and its
// weight are float quantities.  Where float rounding lands on the last
// input sample with a non-zero weight the slope is taken as zero (the
// reference reads one element past its buffer there).
__device__ __forceinline__ float stretch_at(const float* __restrict__ in,
                                            unsigned in_count, unsigned i,
                                            float step)
{
    float x = i * step;
    unsigned int j = x;
    float lo = in[j];
    float hi = (j + 1 < in_count) ? in[j + 1] : lo;
    return lo + ((x - j > 1e-5f) ? (x - j) * (hi - lo) : 0.f);
}

// ---- harmonic sums (reference src/kernels.cu:34-100) ------------------
// Index of fraction m/2^h of bin i: (int)(i*m/2^h + 0.5), exact in
// integer arithmetic.
template <int H>
__device__ __forceinline__ unsigned frac_index(unsigned i, unsigned m)
{
    return (unsigned)(((unsigned long long)i * m + (1u << (H - 1))) >> H);
}

// Sum of `nparts` partials by one warp in a fixed order (lane j adds
// partials j, j+32, ... in turn, then a fixed shuffle tree): deterministic,
// and ~30x shorter than one thread walking the array.  Every lane of the
// warp must call it; all receive the totals.
__device__ __forceinline__ void warp_sum_partials(const double2* __restrict__ partials,
                                                  int nparts, double& a, double& b)
{
    const int lane = threadIdx.x & 31;
    double sa = 0.0, sb = 0.0;
    for (int i = lane; i < nparts; i += 32) {
        const double2 v = partials[i];
        sa += v.x;
        sb += v.y;
    }
    for (int o = 16; o; o >>= 1) {
        sa += __shfl_down_sync(0xffffffffu, sa, o);
        sb += __shfl_down_sync(0xffffffffu, sb, o);
    }
    a = __shfl_sync(0xffffffffu, sa, 0);
    b = __shfl_sync(0xffffffffu, sb, 0);
}

}  // namespace psx
