// psx_kernels.cu -- single-stage kernels behind the drop-in entry points
// of include/peasoup_b200.h (one launch per call, asynchronous).
//
// Layout conventions: time series are float[N]; complex spectra are
// interleaved float pairs (cufftComplex); all grids are grid-stride loops
// sized to a multiple of the SM count (psx::grid_for).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>
#include "psx_common.cuh"
#include "psx_device.cuh"
#include "psx_stages.cuh"

namespace psx {

static thread_local std::string g_err;

void set_error(const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

void clear_error() { g_err.clear(); }

int sm_count()
{
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

// ------------------------------------------------------------------ resample
// Each thread writes four consecutive outputs with one 128-bit store; the
// reads are a near-unit-stride gather that L1/L2 coalesce.
template <bool CENTRED>
__global__ void __launch_bounds__(256) k_resample(const float* __restrict__ in,
                                                  float* __restrict__ out,
                                                  size_t n, double k, double size,
                                                  const double* __restrict__ ktab,
                                                  size_t out_pitch)
{
    const unsigned t = blockIdx.y;
    if (ktab) k = ktab[t];
    float* o = out + (size_t)t * out_pitch;
    const size_t n4 = n / 4;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
        const unsigned long long i0 = 4ull * q;
        float4 v;
        if (CENTRED) {
            double s2 = size * 0.5;
            v.x = gather_at(in, resample_index(i0 + 0, k, s2), n);
            v.y = gather_at(in, resample_index(i0 + 1, k, s2), n);
            v.z = gather_at(in, resample_index(i0 + 2, k, s2), n);
            v.w = gather_at(in, resample_index(i0 + 3, k, s2), n);
        } else {
            const double id = (double)i0;  // exact (n < 2^32)
            v.x = resampleII_read(in, id, k, size, (unsigned)n);
            v.y = resampleII_read(in, id + 1.0, k, size, (unsigned)n);
            v.z = resampleII_read(in, id + 2.0, k, size, (unsigned)n);
            v.w = resampleII_read(in, id + 3.0, k, size, (unsigned)n);
        }
        reinterpret_cast<float4*>(o)[q] = v;
    }
    // tail (n not a multiple of 4)
    if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
        const unsigned long long i = 4ull * n4 + threadIdx.x;
        o[i] = CENTRED ? gather_at(in, resample_index(i, k, size * 0.5), n)
                       : resampleII_read(in, (double)i, k, size, (unsigned)n);
    }
}

double accel_fact(float acc, float tsamp)
{
    // reference src/kernels.cu:361: float product, double divide
    float at = acc * tsamp;
    return (double)at / (2 * 299792458.0);
}

int launch_resample(const float* d_in, float* d_out, size_t n, const double* d_ktab,
                    double k, int ntrials, size_t out_pitch, bool centred, cudaStream_t s)
{
    if (!d_in || !d_out || n == 0 || n >= (size_t(1) << 32) || ntrials <= 0) {
        set_error("resample: bad arguments (1 <= n < 2^32)");
        return PSX_ERR_INVALID;
    }
    const unsigned threads = 256;
    dim3 grid(grid_for((n + 3) / 4, threads, 8), (unsigned)ntrials);
    if (centred)
        k_resample<true><<<grid, threads, 0, s>>>(d_in, d_out, n, k, (double)n, d_ktab, out_pitch);
    else
        k_resample<false><<<grid, threads, 0, s>>>(d_in, d_out, n, k, (double)n, d_ktab, out_pitch);
    return launch_status("resample kernel");
}

// ------------------------------------------------------------------- forming
// way 0 amplitude, way 1 interbinned amplitude.  Each thread forms two
// bins from one 128-bit load of two complex values; bin 2q-1 comes from
// the neighbouring lane (or a cached scalar load at warp edges).
template <int WAY>
__global__ void __launch_bounds__(256) k_form(const float* __restrict__ X,
                                              float* __restrict__ out, size_t nbins)
{
    const size_t npairs = nbins / 2;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += stride) {
        const float4 v = reinterpret_cast<const float4*>(X)[q];
        float2 r;
        if (WAY == 0) {
            r.x = amplitude(v.x, v.y);
            r.y = amplitude(v.z, v.w);
        } else {
            float rl = 0.f, il = 0.f;
            if (q > 0) {
                rl = X[4 * q - 2];
                il = X[4 * q - 1];
            }
            r.x = interbin(v.x, v.y, rl, il);
            r.y = interbin(v.z, v.w, v.x, v.y);
        }
        reinterpret_cast<float2*>(out)[q] = r;
    }
    if ((nbins & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const size_t k = nbins - 1;
        const float re = X[2 * k], im = X[2 * k + 1];
        if (WAY == 0) {
            out[k] = amplitude(re, im);
        } else {
            const float rl = k ? X[2 * k - 2] : 0.f, il = k ? X[2 * k - 1] : 0.f;
            out[k] = interbin(re, im, rl, il);
        }
    }
}

// -------------------------------------------------------------- dereddening
__global__ void __launch_bounds__(256) k_scrunch5(const float* __restrict__ in, size_t count,
                                                  float* __restrict__ out)
{
    if (count < 5) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            float r = 0.f;
            if (count == 1) r = in[0];
            else if (count == 2) r = 0.5f * (in[0] + in[1]);
            else if (count == 3) r = med3(in[0], in[1], in[2]);
            else if (count == 4) r = med4(in[0], in[1], in[2], in[3]);
            if (count) out[0] = r;
        }
        return;
    }
    const size_t oc = count / 5;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < oc; i += stride) {
        const float* p = in + 5 * i;
        out[i] = med5(p[0], p[1], p[2], p[3], p[4]);
    }
}

// Stretch of the three median levels, spliced at pos5/pos25; with X given
// the spectrum is divided by the median in place (bins 0..4 zeroed),
// otherwise the median itself is written.
struct MedianLevels {
    const float* m5;
    const float* m25;
    const float* m125;
    unsigned n5, n25, n125;
    float step5, step25, step125;
    unsigned pos5, pos25;
};

__device__ __forceinline__ float median_at(const MedianLevels& L, unsigned k)
{
    if (k < L.pos5) return stretch_at(L.m5, L.n5, k, L.step5);
    if (k < L.pos25) return stretch_at(L.m25, L.n25, k, L.step25);
    return stretch_at(L.m125, L.n125, k, L.step125);
}

__global__ void __launch_bounds__(256) k_median_apply(MedianLevels L, size_t nbins,
                                                      float* __restrict__ median_out,
                                                      float* __restrict__ X, size_t x_stride = 0,
                                                      size_t m_stride = 0)
{
    if (blockIdx.y) {  // row blockIdx.y of a batch (strides in floats)
        L.m5 += (size_t)blockIdx.y * m_stride;
        L.m25 += (size_t)blockIdx.y * m_stride;
        L.m125 += (size_t)blockIdx.y * m_stride;
        if (X) X += (size_t)blockIdx.y * x_stride;
    }
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nbins; k += stride) {
        const float m = median_at(L, (unsigned)k);
        if (median_out) median_out[k] = m;
        if (X) {
            cuComplex* c = reinterpret_cast<cuComplex*>(X);
            if (k < 5)
                c[k] = make_cuComplex(0.0, 0.0);
            else
                c[k] = cuCdivf(c[k], make_cuComplex(m, 0.0));
        }
    }
}

__global__ void __launch_bounds__(256) k_divide_c_by_f(float* __restrict__ X,
                                                       const float* __restrict__ f, size_t nbins)
{
    cuComplex* c = reinterpret_cast<cuComplex*>(X);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nbins; k += stride) {
        if (k < 5)
            c[k] = make_cuComplex(0.0, 0.0);
        else
            c[k] = cuCdivf(c[k], make_cuComplex(f[k], 0.0));
    }
}

__global__ void __launch_bounds__(256) k_stretch(const float* __restrict__ in, unsigned in_count,
                                                 float* __restrict__ out, size_t out_count,
                                                 float step)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < out_count; i += stride)
        out[i] = stretch_at(in, in_count, (unsigned)i, step);
}

size_t median_scratch_bytes(size_t nbins)
{
    auto up = [](size_t v) { return (v + 63) / 64 * 64; };
    return sizeof(float) * (up(nbins / 5 + 1) + up(nbins / 25 + 1) + up(nbins / 125 + 1));
}

static float stretch_step(size_t in_count, size_t out_count)
{
    // reference src/kernels.cu:1016: float(in_count-1)/(out_count-1)
    return (float)(in_count - 1) / (float)(out_count - 1);
}

// Amplitudes of the complex spectrum X and their three median-of-5
// levels in one pass: a CTA takes groups of 125 bins (5 * 25) at a time, so
// every value of the 5-, 25- and 125-bin levels it writes is formed from
// its own bins; the levels stop where the reference's floor(count / 5)
// stops them.  The amplitudes themselves are never written.
constexpr int kScrGroups = 16;  // 125-bin groups per CTA step

__global__ void __launch_bounds__(256) k_amp_scrunch3(const float* __restrict__ X, size_t nbins,
                                                      float* __restrict__ m5, size_t n5,
                                                      float* __restrict__ m25, size_t n25,
                                                      float* __restrict__ m125, size_t n125,
                                                      size_t x_stride = 0, size_t m_stride = 0)
{
    // row blockIdx.y of a batch: its spectrum and its scratch (strides in floats)
    X += (size_t)blockIdx.y * x_stride;
    m5 += (size_t)blockIdx.y * m_stride;
    m25 += (size_t)blockIdx.y * m_stride;
    m125 += (size_t)blockIdx.y * m_stride;
    __shared__ float s5[kScrGroups * 25];
    __shared__ float s25[kScrGroups * 5];
    const size_t ngroups = (n5 + 24) / 25;  // groups holding any 5-level value
    for (size_t g0 = (size_t)blockIdx.x * kScrGroups; g0 < ngroups;
         g0 += (size_t)gridDim.x * kScrGroups) {
        for (int i = threadIdx.x; i < kScrGroups * 25; i += blockDim.x) {
            const size_t j = g0 * 25 + i;  // 5-level index
            float v = 0.f;
            if (j < n5) {
                const float2* p = reinterpret_cast<const float2*>(X) + 5 * j;
                float a[5];
#pragma unroll
                for (int t = 0; t < 5; ++t) {
                    const float2 z = p[t];
                    a[t] = amplitude(z.x, z.y);
                }
                v = med5(a[0], a[1], a[2], a[3], a[4]);
                m5[j] = v;
            }
            s5[i] = v;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kScrGroups * 5; i += blockDim.x) {
            const size_t j = g0 * 5 + i;
            float v = 0.f;
            if (j < n25) {
                const float* q = s5 + 5 * i;
                v = med5(q[0], q[1], q[2], q[3], q[4]);
                m25[j] = v;
            }
            s25[i] = v;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kScrGroups; i += blockDim.x) {
            const size_t j = g0 + i;
            if (j < n125) {
                const float* q = s25 + 5 * i;
                m125[j] = med5(q[0], q[1], q[2], q[3], q[4]);
            }
        }
        __syncthreads();
    }
}

namespace {

// The stretch, splice and division of launch_running_median once the three
// levels are in the scratch.
int median_apply(size_t nbins, double bin_width, float b5, float b25, float* d_median, float* d_X,
                 float* m5, float* m25, float* m125, cudaStream_t s)
{
    const size_t n5 = nbins / 5, n25 = nbins / 5 / 5, n125 = nbins / 5 / 5 / 5;
    int pos5 = (int)((double)b5 / bin_width);
    int pos25 = (int)((double)b25 / bin_width);
    MedianLevels L;
    L.m5 = m5;
    L.m25 = m25;
    L.m125 = m125;
    L.n5 = (unsigned)n5;
    L.n25 = (unsigned)n25;
    L.n125 = (unsigned)n125;
    L.step5 = stretch_step(n5, nbins);
    L.step25 = stretch_step(n25, nbins);
    L.step125 = stretch_step(n125, nbins);
    L.pos5 = (unsigned)(pos5 < 0 ? 0 : (size_t)pos5 > nbins ? nbins : pos5);
    L.pos25 = (unsigned)(pos25 < 0 ? 0 : (size_t)pos25 > nbins ? nbins : pos25);
    if (L.pos25 < L.pos5) L.pos25 = L.pos5;
    k_median_apply<<<grid_for(nbins, 256), 256, 0, s>>>(L, nbins, d_median, d_X);
    return launch_status("median apply kernel");
}

}  // namespace

int launch_running_median_spectrum(float* d_X, size_t nbins, double bin_width, float b5,
                                   float b25, void* d_scratch, cudaStream_t s)
{
    if (!d_X || !d_scratch || nbins < 125 || nbins > 0xffffffffu) {
        set_error("running median: bad arguments (nbins=%zu)", nbins);
        return PSX_ERR_INVALID;
    }
    auto up = [](size_t v) { return (v + 63) / 64 * 64; };
    float* m5 = static_cast<float*>(d_scratch);
    float* m25 = m5 + up(nbins / 5 + 1);
    float* m125 = m25 + up(nbins / 25 + 1);
    const size_t n5 = nbins / 5, n25 = n5 / 5, n125 = n25 / 5;
    const size_t ngroups = (n5 + 24) / 25;
    const unsigned grid = (unsigned)std::min<size_t>((ngroups + kScrGroups - 1) / kScrGroups,
                                                     (size_t)sm_count() * 8);
    k_amp_scrunch3<<<grid, 256, 0, s>>>(d_X, nbins, m5, n5, m25, n25, m125, n125);
    PSX_TRY(launch_status("amplitude + scrunch kernel"));
    return median_apply(nbins, bin_width, b5, b25, nullptr, d_X, m5, m25, m125, s);
}

int launch_running_median(const float* d_powers, size_t nbins, double bin_width, float b5,
                          float b25, float* d_median, float* d_X, void* d_scratch,
                          cudaStream_t s)
{
    if (!d_powers || !d_scratch || nbins < 125 || nbins > 0xffffffffu) {
        set_error("running median: bad arguments (nbins=%zu)", nbins);
        return PSX_ERR_INVALID;
    }
    auto up = [](size_t v) { return (v + 63) / 64 * 64; };
    float* m5 = static_cast<float*>(d_scratch);
    float* m25 = m5 + up(nbins / 5 + 1);
    float* m125 = m25 + up(nbins / 25 + 1);
    const size_t n5 = nbins / 5, n25 = nbins / 5 / 5, n125 = nbins / 5 / 5 / 5;
    const unsigned T = 256;
    k_scrunch5<<<grid_for(n5, T), T, 0, s>>>(d_powers, nbins, m5);
    k_scrunch5<<<grid_for(n25, T), T, 0, s>>>(m5, n5, m25);
    k_scrunch5<<<grid_for(n125, T), T, 0, s>>>(m25, n25, m125);
    // reference dereddener.hpp:48-49: (int)(boundary / bin_width)
    int pos5 = (int)((double)b5 / bin_width);
    int pos25 = (int)((double)b25 / bin_width);
    MedianLevels L;
    L.m5 = m5;
    L.m25 = m25;
    L.m125 = m125;
    L.n5 = (unsigned)n5;
    L.n25 = (unsigned)n25;
    L.n125 = (unsigned)n125;
    L.step5 = stretch_step(n5, nbins);
    L.step25 = stretch_step(n25, nbins);
    L.step125 = stretch_step(n125, nbins);
    L.pos5 = (unsigned)(pos5 < 0 ? 0 : (size_t)pos5 > nbins ? nbins : pos5);
    L.pos25 = (unsigned)(pos25 < 0 ? 0 : (size_t)pos25 > nbins ? nbins : pos25);
    if (L.pos25 < L.pos5) L.pos25 = L.pos5;
    k_median_apply<<<grid_for(nbins, T), T, 0, s>>>(L, nbins, d_median, d_X);
    return launch_status("running median kernels");
}

// ------------------------------------------------------------------- zapping
// One warp per birdie; lanes stride the birdie's bin range.
__global__ void k_zap(float* __restrict__ X, const float* __restrict__ freqs,
                      const float* __restrict__ widths, float bin_width, unsigned nbirdies,
                      unsigned nbins, size_t x_stride = 0)
{
    X += (size_t)blockIdx.y * x_stride;  // row blockIdx.y of a batch
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const unsigned lane = threadIdx.x & 31;
    if (warp >= nbirdies) return;
    const float freq = freqs[warp];
    const float width = widths[warp];
    int low_bin = __float2int_rd((freq - width) / bin_width);
    int high_bin = __float2int_ru((freq + width) / bin_width);
    if (low_bin < 0) low_bin = 0;
    if (low_bin >= (int)nbins) return;
    if (high_bin >= (int)nbins) high_bin = (int)nbins - 1;
    float2* c = reinterpret_cast<float2*>(X);
    for (int k = low_bin + (int)lane; k < high_bin; k += 32) c[k] = make_float2(1.0f, 0.0f);
}

int launch_zap(float* d_X, const float* d_freqs, const float* d_widths, float bin_width,
               size_t nbirdies, size_t nbins, cudaStream_t s)
{
    if (nbirdies == 0) return PSX_OK;
    if (!d_X || !d_freqs || !d_widths) {
        set_error("zap: null pointer");
        return PSX_ERR_INVALID;
    }
    const unsigned T = 256;
    const unsigned blocks = (unsigned)((nbirdies * 32 + T - 1) / T);
    k_zap<<<blocks, T, 0, s>>>(d_X, d_freqs, d_widths, bin_width, (unsigned)nbirdies,
                               (unsigned)nbins);
    return launch_status("zap kernel");
}

// ---------------------------------------------------------------- reductions
// Deterministic two-level sum of x and x^2 (double accumulators): each
// block writes its partials, one block adds them in fixed order.
template <class Src>
__global__ void __launch_bounds__(256) k_sum_partials(Src src, size_t first, size_t n,
                                                      double2* __restrict__ partials)
{
    double s = 0.0, s2 = 0.0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = first + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double v = src(i);
        s += v;
        s2 += v * v;
    }
    for (int o = 16; o; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    __shared__ double sh[2][8];
    const int w = threadIdx.x / 32;
    if ((threadIdx.x & 31) == 0) {
        sh[0][w] = s;
        sh[1][w] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); ++i) {
            a += sh[0][i];
            b += sh[1][i];
        }
        partials[blockIdx.x] = make_double2(a, b);
    }
}

// Adds `nparts` partials (one warp, fixed order); writes the totals to sums[0..1]
// and, when stat != nullptr, the reference's float statistics
// {mean, rms, std, mean*scale, std*scale} computed exactly as its host
// code does (stats.hpp:20-31 and src/kernels.cu:443,458), without
// contraction.
__global__ void k_finish_stats(const double2* __restrict__ partials, int nparts, double count,
                               double* __restrict__ sums, float* __restrict__ stat, float scale,
                               size_t part_stride = 0, size_t sums_stride = 0,
                               size_t stat_stride = 0)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    // row blockIdx.y of a batch (strides in elements)
    partials += (size_t)blockIdx.y * part_stride;
    sums += (size_t)blockIdx.y * sums_stride;
    if (stat) stat += (size_t)blockIdx.y * stat_stride;
    double a, b;
    warp_sum_partials(partials, nparts, a, b);
    if (threadIdx.x != 0) return;
    sums[0] = a;
    sums[1] = b;
    if (stat) {
        const float cnt = (float)count;
        const float mean = __fdiv_rn((float)a, cnt);
        const float rms = sqrtf(__fdiv_rn((float)b, cnt));
        const float sd = sqrtf(__fsub_rn(__fmul_rn(rms, rms), __fmul_rn(mean, mean)));
        stat[0] = mean;
        stat[1] = rms;
        stat[2] = sd;
        stat[3] = __fmul_rn(mean, scale);
        stat[4] = __fmul_rn(sd, scale);
    }
}

struct PlainSrc {
    const float* x;
    __device__ double operator()(size_t i) const { return (double)x[i]; }
};

struct InterbinSrc {
    const float* X;
    __device__ double operator()(size_t k) const
    {
        const float re = X[2 * k], im = X[2 * k + 1];
        const float rl = k ? X[2 * k - 2] : 0.f, il = k ? X[2 * k - 1] : 0.f;
        return (double)interbin(re, im, rl, il);
    }
};

// Block sum of (a, b) pairs into partials[blockIdx.x] (fixed order).
template <int NT>
__device__ __forceinline__ void block_partials(double s, double s2, double2* __restrict__ partials)
{
    for (int o = 16; o; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    __shared__ double sh[2][NT / 32];
    const int w = threadIdx.x / 32;
    if ((threadIdx.x & 31) == 0) {
        sh[0][w] = s;
        sh[1][w] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < NT / 32; ++i) {
            a += sh[0][i];
            b += sh[1][i];
        }
        partials[blockIdx.x] = make_double2(a, b);
    }
}

__device__ __forceinline__ void acc4(float4 v, double& s, double& s2)
{
    const double a = v.x, b = v.y, c = v.z, d = v.w;
    s += (a + b) + (c + d);
    s2 += (a * a + b * b) + (c * c + d * d);
}

constexpr int kVecThreads = 512;

// Partial sums of x and x^2 over [0, n) with 128-bit loads (x 16-byte
// aligned); the n % 4 tail is added by block 0.  With `copy` set, x is also
// written there (16-byte aligned), fusing the copy of a series into its
// first pass; with `state` set, block 0 starts the baseline loop state
// (state[0] = 1 active, state[1] = 0 passes).
__global__ void __launch_bounds__(kVecThreads) k_partials_v4(const float* __restrict__ x, size_t n,
                                                             double2* __restrict__ partials,
                                                             float* __restrict__ copy,
                                                             unsigned* __restrict__ state,
                                                             size_t x_stride = 0,
                                                             size_t part_stride = 0,
                                                             size_t state_stride = 0)
{
    // row blockIdx.y of a batch (strides in elements; no copy in a batch)
    x += (size_t)blockIdx.y * x_stride;
    partials += (size_t)blockIdx.y * part_stride;
    if (state) state += (size_t)blockIdx.y * state_stride;
    if (state && blockIdx.x == 0 && threadIdx.x == 0) {
        state[0] = 1u;
        state[1] = 0u;
    }
    double s = 0.0, s2 = 0.0;
    const size_t n4 = n / 4, stride = (size_t)gridDim.x * blockDim.x;
    const float4* x4 = reinterpret_cast<const float4*>(x);
    float4* c4 = reinterpret_cast<float4*>(copy);
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
        const float4 v = x4[q];
        if (copy) c4[q] = v;
        acc4(v, s, s2);
    }
    if (blockIdx.x == 0 && threadIdx.x < n - 4 * n4) {
        const float v = x[4 * n4 + threadIdx.x];
        if (copy) copy[4 * n4 + threadIdx.x] = v;
        s += (double)v;
        s2 += (double)v * v;
    }
    block_partials<kVecThreads>(s, s2, partials);
}

// One pass of the device-side baseline loop (reference src/kernels.cu:
// 463-479) in one kernel.  While *flag_in says the loop goes on, every CTA
// forms the float mean of the previous pass's partials (float sum / float
// count; the same fixed-order sum in every CTA), subtracts it, and, while
// |mean| > 5e-7 n, writes its partials of the new x to part_out; CTA 0
// records the decision in *flag_out and counts the pass.  Flags and
// partials alternate between passes, so no CTA reads what this pass writes.
// With fin_flag set (the last pass) the final decision and the pass count
// are copied there and to fin_passes.
__global__ void __launch_bounds__(kVecThreads) k_baseline_pass_v4(
    float* __restrict__ x, size_t n, double count, const double2* __restrict__ part_in,
    int nparts, double2* __restrict__ part_out, const unsigned* __restrict__ flag_in,
    unsigned* __restrict__ flag_out, unsigned* __restrict__ passes,
    unsigned* __restrict__ fin_flag, unsigned* __restrict__ fin_passes, size_t x_stride = 0,
    size_t part_stride = 0, size_t flag_stride = 0)
{
    if (blockIdx.y) {  // row blockIdx.y of a batch (strides in elements)
        const size_t r = blockIdx.y;
        x += r * x_stride;
        part_in += r * part_stride;
        part_out += r * part_stride;
        flag_in += r * flag_stride;
        flag_out += r * flag_stride;
        passes += r * flag_stride;
        if (fin_flag) fin_flag += r * flag_stride;
        if (fin_passes) fin_passes += r * flag_stride;
    }
    __shared__ float s_mean;
    __shared__ int s_go;
    if (*flag_in == 0u) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            *flag_out = 0u;
            if (fin_flag) {
                *fin_flag = 0u;
                *fin_passes = *passes;
            }
        }
        return;
    }
    if (threadIdx.x < 32) {
        double a, b;
        warp_sum_partials(part_in, nparts, a, b);
        if (threadIdx.x == 0) {
            const float mean = __fdiv_rn((float)a, (float)count);
            s_mean = mean;
            s_go = (fabsf(mean) > 5e-7 * count) ? 1 : 0;
        }
    }
    __syncthreads();
    const float m = s_mean;
    const bool sum = s_go != 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned np = *passes + 1u;
        *passes = np;
        *flag_out = sum ? 1u : 0u;
        if (fin_flag) {
            *fin_flag = sum ? 1u : 0u;
            *fin_passes = np;
        }
    }
    if (m == 0.0f) return;
    double s = 0.0, s2 = 0.0;
    const size_t n4 = n / 4, stride = (size_t)gridDim.x * blockDim.x;
    float4* x4 = reinterpret_cast<float4*>(x);
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
        float4 v = x4[q];
        v.x -= m;
        v.y -= m;
        v.z -= m;
        v.w -= m;
        x4[q] = v;
        if (sum) acc4(v, s, s2);
    }
    if (blockIdx.x == 0 && threadIdx.x < n - 4 * n4) {
        const float v = x[4 * n4 + threadIdx.x] - m;
        x[4 * n4 + threadIdx.x] = v;
        s += (double)v;
        s2 += (double)v * v;
    }
    if (sum) block_partials<kVecThreads>(s, s2, part_out);
}

// Partial sums of the interbinned amplitude of the complex spectrum X over
// bins [0, nbins): two bins per thread from one 128-bit load, the previous
// bin's pair from a 64-bit load; the odd last bin is added by block 0.
__global__ void __launch_bounds__(kVecThreads) k_interbin_partials_v4(const float* __restrict__ X,
                                                                      size_t nbins,
                                                                      double2* __restrict__ partials,
                                                                      size_t x_stride = 0,
                                                                      size_t part_stride = 0)
{
    X += (size_t)blockIdx.y * x_stride;  // row blockIdx.y of a batch
    partials += (size_t)blockIdx.y * part_stride;
    double s = 0.0, s2 = 0.0;
    const size_t npairs = nbins / 2, stride = (size_t)gridDim.x * blockDim.x;
    const float4* X4 = reinterpret_cast<const float4*>(X);
    const float2* X2 = reinterpret_cast<const float2*>(X);
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += stride) {
        const float4 v = X4[q];
        const float2 l = q ? X2[2 * q - 1] : make_float2(0.f, 0.f);
        const double a = interbin(v.x, v.y, l.x, l.y);
        const double b = interbin(v.z, v.w, v.x, v.y);
        s += a + b;
        s2 += a * a + b * b;
    }
    if ((nbins & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const size_t k = nbins - 1;
        const float2 l = k ? X2[k - 1] : make_float2(0.f, 0.f);
        const double a = interbin(X[2 * k], X[2 * k + 1], l.x, l.y);
        s += a;
        s2 += a * a;
    }
    block_partials<kVecThreads>(s, s2, partials);
}

int reduction_blocks() { return sm_count() * 2; }

int launch_partials_v4(const float* d_x, size_t n, double2* d_partials, float* d_copy,
                       unsigned* d_state, cudaStream_t s)
{
    k_partials_v4<<<reduction_blocks(), kVecThreads, 0, s>>>(d_x, n, d_partials, d_copy, d_state);
    return launch_status("partial sums kernel");
}

int launch_baseline_pass_v4(float* d_x, size_t n, const double2* d_part_in, double2* d_part_out,
                            const unsigned* d_flag_in, unsigned* d_flag_out, unsigned* d_passes,
                            unsigned* d_fin_flag, unsigned* d_fin_passes, cudaStream_t s)
{
    const int nb = reduction_blocks();
    k_baseline_pass_v4<<<nb, kVecThreads, 0, s>>>(d_x, n, (double)n, d_part_in, nb, d_part_out,
                                                  d_flag_in, d_flag_out, d_passes, d_fin_flag,
                                                  d_fin_passes);
    return launch_status("baseline pass kernel");
}

int launch_interbin_stats_v4(const float* d_X, size_t nbins, double2* d_partials, double* d_sums,
                             float* d_stat, float scale, cudaStream_t s)
{
    const int nb = reduction_blocks();
    k_interbin_partials_v4<<<nb, kVecThreads, 0, s>>>(d_X, nbins, d_partials);
    k_finish_stats<<<1, 32, 0, s>>>(d_partials, nb, (double)nbins, d_sums, d_stat, scale);
    return launch_status("interbin statistics kernels");
}

// ---- row-batched prologue stages (the grouped prologue of the engine)
int launch_partials_rows(const float* d_x, size_t n, size_t x_stride, int rows,
                         double2* d_partials, size_t part_stride, unsigned* d_state,
                         size_t state_stride, cudaStream_t s)
{
    if (rows < 1 || rows > 65535) {
        set_error("partial sums: bad row count %d", rows);
        return PSX_ERR_INVALID;
    }
    k_partials_v4<<<dim3(reduction_blocks(), rows), kVecThreads, 0, s>>>(
        d_x, n, d_partials, nullptr, d_state, x_stride, part_stride, state_stride);
    return launch_status("partial sums kernel (rows)");
}

int launch_baseline_pass_rows(float* d_x, size_t n, size_t x_stride, int rows,
                              const double2* d_part_in, double2* d_part_out, size_t part_stride,
                              const unsigned* d_flag_in, unsigned* d_flag_out,
                              unsigned* d_passes, unsigned* d_fin_flag, unsigned* d_fin_passes,
                              size_t flag_stride, cudaStream_t s)
{
    const int nb = reduction_blocks();
    k_baseline_pass_v4<<<dim3(nb, rows), kVecThreads, 0, s>>>(
        d_x, n, (double)n, d_part_in, nb, d_part_out, d_flag_in, d_flag_out, d_passes, d_fin_flag,
        d_fin_passes, x_stride, part_stride, flag_stride);
    return launch_status("baseline pass kernel (rows)");
}

int launch_running_median_spectrum_rows(float* d_X, size_t x_stride, int rows, size_t nbins,
                                        double bin_width, float b5, float b25, void* d_scratch,
                                        size_t scratch_stride_floats, cudaStream_t s)
{
    if (!d_X || !d_scratch || nbins < 125 || nbins > 0xffffffffu) {
        set_error("running median: bad arguments (nbins=%zu)", nbins);
        return PSX_ERR_INVALID;
    }
    auto up = [](size_t v) { return (v + 63) / 64 * 64; };
    float* m5 = static_cast<float*>(d_scratch);
    float* m25 = m5 + up(nbins / 5 + 1);
    float* m125 = m25 + up(nbins / 25 + 1);
    const size_t n5 = nbins / 5, n25 = n5 / 5, n125 = n25 / 5;
    const size_t ngroups = (n5 + 24) / 25;
    const unsigned grid = (unsigned)std::min<size_t>((ngroups + kScrGroups - 1) / kScrGroups,
                                                     (size_t)sm_count() * 8);
    k_amp_scrunch3<<<dim3(grid, rows), 256, 0, s>>>(d_X, nbins, m5, n5, m25, n25, m125, n125,
                                                     x_stride, scratch_stride_floats);
    PSX_TRY(launch_status("amplitude + scrunch kernel (rows)"));
    int pos5 = (int)((double)b5 / bin_width);
    int pos25 = (int)((double)b25 / bin_width);
    MedianLevels L;
    L.m5 = m5;
    L.m25 = m25;
    L.m125 = m125;
    L.n5 = (unsigned)n5;
    L.n25 = (unsigned)n25;
    L.n125 = (unsigned)n125;
    L.step5 = stretch_step(n5, nbins);
    L.step25 = stretch_step(n25, nbins);
    L.step125 = stretch_step(n125, nbins);
    L.pos5 = (unsigned)(pos5 < 0 ? 0 : (size_t)pos5 > nbins ? nbins : pos5);
    L.pos25 = (unsigned)(pos25 < 0 ? 0 : (size_t)pos25 > nbins ? nbins : pos25);
    if (L.pos25 < L.pos5) L.pos25 = L.pos5;
    k_median_apply<<<dim3(grid_for(nbins, 256), rows), 256, 0, s>>>(
        L, nbins, nullptr, d_X, x_stride, scratch_stride_floats);
    return launch_status("median apply kernel (rows)");
}

int launch_zap_rows(float* d_X, size_t x_stride, int rows, const float* d_freqs,
                    const float* d_widths, float bin_width, size_t nbirdies, size_t nbins,
                    cudaStream_t s)
{
    if (nbirdies == 0) return PSX_OK;
    if (!d_X || !d_freqs || !d_widths) {
        set_error("zap: null pointer");
        return PSX_ERR_INVALID;
    }
    const unsigned T = 256;
    const unsigned blocks = (unsigned)((nbirdies * 32 + T - 1) / T);
    k_zap<<<dim3(blocks, rows), T, 0, s>>>(d_X, d_freqs, d_widths, bin_width, (unsigned)nbirdies,
                                          (unsigned)nbins, x_stride);
    return launch_status("zap kernel (rows)");
}

int launch_interbin_stats_rows(const float* d_X, size_t x_stride, int rows, size_t nbins,
                               double2* d_partials, size_t part_stride, double* d_sums,
                               size_t sums_stride, float* d_stat, size_t stat_stride, float scale,
                               cudaStream_t s)
{
    const int nb = reduction_blocks();
    k_interbin_partials_v4<<<dim3(nb, rows), kVecThreads, 0, s>>>(d_X, nbins, d_partials, x_stride,
                                                                  part_stride);
    k_finish_stats<<<dim3(1, rows), 32, 0, s>>>(d_partials, nb, (double)nbins, d_sums, d_stat,
                                                scale, part_stride, sums_stride, stat_stride);
    return launch_status("interbin statistics kernels (rows)");
}

int launch_partials(const float* d_x, size_t n, double2* d_partials, cudaStream_t s)
{
    k_sum_partials<PlainSrc><<<reduction_blocks(), 256, 0, s>>>(PlainSrc{d_x}, 0, n, d_partials);
    return launch_status("partial sums kernel");
}

int launch_stats(const float* d_x, bool interbinned, size_t first, size_t n, double2* d_partials,
                 double* d_sums, float* d_stat, float scale, cudaStream_t s)
{
    const unsigned T = 256;
    const int nb = reduction_blocks();
    if (interbinned)
        k_sum_partials<InterbinSrc><<<nb, T, 0, s>>>(InterbinSrc{d_x}, first, n, d_partials);
    else
        k_sum_partials<PlainSrc><<<nb, T, 0, s>>>(PlainSrc{d_x}, first, n, d_partials);
    k_finish_stats<<<1, 32, 0, s>>>(d_partials, nb, (double)(n - first), d_sums, d_stat, scale);
    return launch_status("statistics kernels");
}

// ------------------------------------------------------------- element-wise
__global__ void k_normalise(float* __restrict__ x, float mean, float sigma, size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        x[i] = normalise(x[i], mean, sigma);
}

__global__ void k_sub_scalar(float* __restrict__ x, size_t n, const float* __restrict__ v)
{
    const float m = *v;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] -= m;
}

__global__ void k_fill(float* __restrict__ x, size_t n, float value, size_t x_stride = 0)
{
    x += (size_t)blockIdx.y * x_stride;  // row blockIdx.y of a batch
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] = value;
}

template <class T>
__global__ void k_convert(const T* __restrict__ in, float* __restrict__ out, size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = static_cast<float>(in[i]);
}

int launch_sub_scalar(float* d_x, size_t n, const float* d_v, cudaStream_t s)
{
    if (n == 0) return PSX_OK;
    k_sub_scalar<<<grid_for(n, 256), 256, 0, s>>>(d_x, n, d_v);
    return launch_status("subtract kernel");
}

int launch_fill(float* d_x, size_t n, float value, cudaStream_t s)
{
    if (n == 0) return PSX_OK;
    k_fill<<<grid_for(n, 256), 256, 0, s>>>(d_x, n, value);
    return launch_status("fill kernel");
}

int launch_fill_rows(float* d_x, size_t n, size_t x_stride, int rows, float value,
                     cudaStream_t s)
{
    if (n == 0) return PSX_OK;
    dim3 grid(grid_for(n, 256), rows);
    k_fill<<<grid, 256, 0, s>>>(d_x, n, value, x_stride);
    return launch_status("fill kernel (rows)");
}

// Mean of d_x[0..n) in float as the reference forms it (float sum / float
// count), from a double-accumulated sum; written to d_mean.
__global__ void k_mean_from_sums(const double* __restrict__ sums, double count,
                                 float* __restrict__ d_mean)
{
    *d_mean = __fdiv_rn((float)sums[0], (float)count);
}

int remove_baseline_pass(float* d_x, size_t n, double2* d_partials, double* d_sums,
                         float* d_mean, cudaStream_t s)
{
    const unsigned T = 256;
    const int nb = reduction_blocks();
    k_sum_partials<PlainSrc><<<nb, T, 0, s>>>(PlainSrc{d_x}, 0, n, d_partials);
    k_finish_stats<<<1, 32, 0, s>>>(d_partials, nb, (double)n, d_sums, nullptr, 0.f);
    k_mean_from_sums<<<1, 1, 0, s>>>(d_sums, (double)n, d_mean);
    k_sub_scalar<<<grid_for(n, T), T, 0, s>>>(d_x, n, d_mean);
    return launch_status("baseline kernels");
}

// ----------------------------------------------------------- harmonic sums
struct FoldPtrs {
    float* p[5];
};

// One thread per output bin, the running sum in the reference's order
// (src/kernels.cu:41-96).
__global__ void __launch_bounds__(256) k_harmonic_sum(const float* __restrict__ in,
                                                      FoldPtrs out, unsigned n, int nharms)
{
    const unsigned stride = gridDim.x * blockDim.x;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float val = in[i];
        if (nharms > 0) {
            val += in[frac_index<1>(i, 1)];
            out.p[0][i] = val * rsqrt(2.0);
        }
        if (nharms > 1) {
            val += in[frac_index<2>(i, 3)];
            val += in[frac_index<2>(i, 1)];
            out.p[1][i] = val * 0.5;
        }
        if (nharms > 2) {
#pragma unroll
            for (unsigned m = 1; m < 8; m += 2) val += in[frac_index<3>(i, m)];
            out.p[2][i] = val * rsqrt(8.0);
        }
        if (nharms > 3) {
#pragma unroll
            for (unsigned m = 1; m < 16; m += 2) val += in[frac_index<4>(i, m)];
            out.p[3][i] = val * 0.25;
        }
        if (nharms > 4) {
#pragma unroll
            for (unsigned m = 1; m < 32; m += 2) val += in[frac_index<5>(i, m)];
            out.p[4][i] = val * rsqrt(32.0);
        }
    }
}

// ------------------------------------------------------------- compaction
// Order-preserving stream compaction of (i, x[i]) with x[i] > thresh over
// [start, n): per-tile counts, a single-block scan, then the scatter.
constexpr int kCompactTile = 4096;

__global__ void __launch_bounds__(256) k_compact_count(const float* __restrict__ x, int start,
                                                       int n, float thresh, int* __restrict__ counts)
{
    const int t0 = start + blockIdx.x * kCompactTile;
    int c = 0;
    for (int i = t0 + threadIdx.x; i < n && i < t0 + kCompactTile; i += blockDim.x)
        c += x[i] > thresh;
    for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ int sh[8];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x / 32] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) s += sh[w];
        counts[blockIdx.x] = s;
    }
}

__global__ void k_compact_scan(int* __restrict__ counts, int ntiles, int* __restrict__ total)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int s = 0;
    for (int i = 0; i < ntiles; ++i) {
        const int c = counts[i];
        counts[i] = s;
        s += c;
    }
    *total = s;
}

__global__ void __launch_bounds__(256) k_compact_write(const float* __restrict__ x, int start,
                                                       int n, float thresh,
                                                       const int* __restrict__ offsets,
                                                       int* __restrict__ idx, float* __restrict__ val,
                                                       int cap)
{
    // one tile per block, processed in order by the block's warps in turn
    const int t0 = start + blockIdx.x * kCompactTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x / 32, nw = blockDim.x / 32;
    __shared__ int warp_base[8];
    __shared__ int running;
    if (threadIdx.x == 0) running = offsets[blockIdx.x];
    __syncthreads();
    for (int c0 = t0; c0 < t0 + kCompactTile && c0 < n; c0 += (int)blockDim.x) {
        const int i = c0 + threadIdx.x;
        const bool hit = i < n && i < t0 + kCompactTile && x[i] > thresh;
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) warp_base[warp] = __popc(m);
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = running;
            for (int w = 0; w < nw; ++w) {
                const int c = warp_base[w];
                warp_base[w] = s;
                s += c;
            }
            running = s;
        }
        __syncthreads();
        if (hit) {
            const int pos = warp_base[warp] + __popc(m & ((1u << lane) - 1));
            if (pos < cap) {
                idx[pos] = i;
                val[pos] = x[i];
            }
        }
        __syncthreads();
    }
}

}  // namespace psx

using namespace psx;

// =================================================================== C ABI
extern "C" {

const char* psx_last_error(void) { return psx::g_err.c_str(); }

const char* psx_status_string(int st)
{
    switch (st) {
    case PSX_OK: return "ok";
    case PSX_ERR_INVALID: return "invalid argument";
    case PSX_ERR_CUDA: return "CUDA error";
    case PSX_ERR_CUFFT: return "cuFFT error";
    case PSX_ERR_ALLOC: return "allocation failed";
    case PSX_ERR_OVERFLOW: return "output buffer too small";
    case PSX_ERR_UNSUPPORTED: return "unsupported";
    case PSX_ERR_IO: return "I/O error";
    case PSX_ERR_BUSY: return "busy";
    default: return "unknown status";
    }
}

const char* psx_version(void) { return "peasoup_b200 0.1 (sm_100a)"; }

int psx_resampleII(const float* d_in, float* d_out, size_t size, float acc, float tsamp,
                   psx_stream_t stream)
{
    clear_error();
    return launch_resample(d_in, d_out, size, nullptr, accel_fact(acc, tsamp), 1, size, false,
                           cs(stream));
}

int psx_resample(const float* d_in, float* d_out, size_t size, float acc, float tsamp,
                 psx_stream_t stream)
{
    clear_error();
    return launch_resample(d_in, d_out, size, nullptr, accel_fact(acc, tsamp), 1, size, true,
                           cs(stream));
}

int psx_resampleII_batch(const float* d_in, float* d_out, size_t size, const float* h_accs,
                         int ntrials, float tsamp, psx_stream_t stream)
{
    clear_error();
    if (!h_accs || ntrials <= 0 || ntrials > 65535) {
        set_error("resampleII_batch: bad trial list");
        return PSX_ERR_INVALID;
    }
    std::vector<double> k(ntrials);
    for (int t = 0; t < ntrials; ++t) k[t] = accel_fact(h_accs[t], tsamp);
    double* d_k = nullptr;
    PSX_CUDA(cudaMallocAsync((void**)&d_k, sizeof(double) * ntrials, cs(stream)));
    int rc = cuda_status(cudaMemcpyAsync(d_k, k.data(), sizeof(double) * ntrials,
                                         cudaMemcpyHostToDevice, cs(stream)),
                         "resampleII_batch copy");
    if (rc == PSX_OK)
        rc = launch_resample(d_in, d_out, size, d_k, 0.0, ntrials, size, false, cs(stream));
    cudaFreeAsync(d_k, cs(stream));
    // the host vector must outlive the copy
    if (rc == PSX_OK) rc = cuda_status(cudaStreamSynchronize(cs(stream)), "resampleII_batch");
    return rc;
}

int psx_form_power_series(const float* d_fseries, float* d_out, size_t nbins, int way,
                          psx_stream_t stream)
{
    clear_error();
    if (!d_fseries || !d_out || nbins == 0 || (way != 0 && way != 1)) {
        set_error("form_power_series: bad arguments");
        return PSX_ERR_INVALID;
    }
    const unsigned T = 256;
    const unsigned g = grid_for(nbins / 2 + 1, T);
    if (way == 0)
        k_form<0><<<g, T, 0, cs(stream)>>>(d_fseries, d_out, nbins);
    else
        k_form<1><<<g, T, 0, cs(stream)>>>(d_fseries, d_out, nbins);
    return launch_status("form kernel");
}

int psx_median_scrunch5(const float* d_in, size_t count, float* d_out, psx_stream_t stream)
{
    clear_error();
    if (!d_in || !d_out || count == 0) {
        set_error("median_scrunch5: bad arguments");
        return PSX_ERR_INVALID;
    }
    k_scrunch5<<<grid_for(count / 5 + 1, 256), 256, 0, cs(stream)>>>(d_in, count, d_out);
    return launch_status("scrunch kernel");
}

int psx_linear_stretch(const float* d_in, size_t in_count, float* d_out, size_t out_count,
                       psx_stream_t stream)
{
    clear_error();
    if (!d_in || !d_out || in_count == 0 || out_count < 2 || in_count > 0xffffffffu ||
        out_count > 0xffffffffu) {
        set_error("linear_stretch: bad arguments");
        return PSX_ERR_INVALID;
    }
    k_stretch<<<grid_for(out_count, 256), 256, 0, cs(stream)>>>(
        d_in, (unsigned)in_count, d_out, out_count, stretch_step(in_count, out_count));
    return launch_status("stretch kernel");
}

size_t psx_running_median_scratch_bytes(size_t nbins) { return median_scratch_bytes(nbins); }

int psx_running_median(const float* d_powers, size_t nbins, double bin_width, float b5,
                       float b25, float* d_median, void* d_scratch, psx_stream_t stream)
{
    clear_error();
    if (!d_median) {
        set_error("running_median: null output");
        return PSX_ERR_INVALID;
    }
    return launch_running_median(d_powers, nbins, bin_width, b5, b25, d_median, nullptr,
                                 d_scratch, cs(stream));
}

int psx_divide_c_by_f(float* d_fseries, const float* d_f, size_t nbins, psx_stream_t stream)
{
    clear_error();
    if (!d_fseries || !d_f || nbins == 0) {
        set_error("divide_c_by_f: bad arguments");
        return PSX_ERR_INVALID;
    }
    k_divide_c_by_f<<<grid_for(nbins, 256), 256, 0, cs(stream)>>>(d_fseries, d_f, nbins);
    return launch_status("divide kernel");
}

int psx_deredden(float* d_fseries, const float* d_powers, size_t nbins, double bin_width,
                 float b5, float b25, void* d_scratch, psx_stream_t stream)
{
    clear_error();
    if (!d_fseries) {
        set_error("deredden: null spectrum");
        return PSX_ERR_INVALID;
    }
    return launch_running_median(d_powers, nbins, bin_width, b5, b25, nullptr, d_fseries,
                                 d_scratch, cs(stream));
}

int psx_zap_birdies(float* d_fseries, const float* d_freqs, const float* d_widths,
                    float bin_width, size_t nbirdies, size_t nbins, psx_stream_t stream)
{
    clear_error();
    return launch_zap(d_fseries, d_freqs, d_widths, bin_width, nbirdies, nbins, cs(stream));
}

int psx_read_zaplist(const char* path, float* h_freqs, float* h_widths, size_t cap, size_t* n)
{
    clear_error();
    if (!path || !n) {
        set_error("read_zaplist: null argument");
        return PSX_ERR_INVALID;
    }
    std::ifstream f(path);
    if (!f.good()) {
        set_error("zap list %s could not be opened", path);
        return PSX_ERR_IO;
    }
    // birdiezapper.hpp:35-46: whitespace-separated "freq width" per line,
    // blank lines skipped, numbers parsed as atof does.
    std::string line;
    size_t k = 0;
    while (std::getline(f, line)) {
        std::istringstream ss(line);
        std::string a, b;
        if (!(ss >> a)) continue;
        if (!(ss >> b)) {
            set_error("zap list %s: line without a width: '%s'", path, line.c_str());
            return PSX_ERR_IO;
        }
        if (h_freqs && k < cap) {
            h_freqs[k] = (float)atof(a.c_str());
            h_widths[k] = (float)atof(b.c_str());
        }
        ++k;
    }
    *n = k;
    if (h_freqs && k > cap) {
        set_error("zap list has %zu entries, buffer holds %zu", k, cap);
        return PSX_ERR_OVERFLOW;
    }
    return PSX_OK;
}

int psx_stats(const float* d_x, size_t n, size_t first, float* h_mean, float* h_rms,
              float* h_std, psx_stream_t stream)
{
    clear_error();
    if (!d_x || n <= first) {
        set_error("stats: bad arguments");
        return PSX_ERR_INVALID;
    }
    cudaStream_t s = cs(stream);
    void* scratch = nullptr;
    const int nb = reduction_blocks();
    const size_t bytes = sizeof(double2) * nb + 2 * sizeof(double) + 8 * sizeof(float);
    PSX_CUDA(cudaMallocAsync(&scratch, bytes, s));
    double2* part = static_cast<double2*>(scratch);
    double* sums = reinterpret_cast<double*>(part + nb);
    float* stat = reinterpret_cast<float*>(sums + 2);
    int rc = launch_stats(d_x, false, first, n, part, sums, stat, 1.0f, s);
    float h[5] = {0, 0, 0, 0, 0};
    if (rc == PSX_OK)
        rc = cuda_status(cudaMemcpyAsync(h, stat, sizeof h, cudaMemcpyDeviceToHost, s), "stats copy");
    cudaFreeAsync(scratch, s);
    if (rc == PSX_OK) rc = cuda_status(cudaStreamSynchronize(s), "stats");
    if (rc == PSX_OK) {
        if (h_mean) *h_mean = h[0];
        if (h_rms) *h_rms = h[1];
        if (h_std) *h_std = h[2];
    }
    return rc;
}

int psx_normalise(float* d_x, float mean, float sigma, size_t n, psx_stream_t stream)
{
    clear_error();
    if (!d_x) {
        set_error("normalise: null pointer");
        return PSX_ERR_INVALID;
    }
    if (n == 0) return PSX_OK;
    k_normalise<<<grid_for(n, 256), 256, 0, cs(stream)>>>(d_x, mean, sigma, n);
    return launch_status("normalise kernel");
}

int psx_remove_baseline(float* d_x, size_t n, int* h_passes, psx_stream_t stream)
{
    clear_error();
    if (!d_x || n == 0) {
        set_error("remove_baseline: bad arguments");
        return PSX_ERR_INVALID;
    }
    cudaStream_t s = cs(stream);
    const int nb = reduction_blocks();
    void* scratch = nullptr;
    PSX_CUDA(cudaMallocAsync(&scratch, sizeof(double2) * nb + 2 * sizeof(double) + 16, s));
    double2* part = static_cast<double2*>(scratch);
    double* sums = reinterpret_cast<double*>(part + nb);
    float* d_mean = reinterpret_cast<float*>(sums + 2);
    int rc = PSX_OK, count = 0;
    float mean = 0.f;
    // reference src/kernels.cu:467-477: do { subtract mean } while
    // (|mean| > 5e-7 n), leaving after the 102nd pass at most.
    do {
        rc = remove_baseline_pass(d_x, n, part, sums, d_mean, s);
        if (rc != PSX_OK) break;
        rc = cuda_status(cudaMemcpyAsync(&mean, d_mean, sizeof(float), cudaMemcpyDeviceToHost, s),
                         "baseline copy");
        if (rc == PSX_OK) rc = cuda_status(cudaStreamSynchronize(s), "baseline");
        if (rc != PSX_OK) break;
        if (count++ > 100) break;
    } while (std::fabs(mean) > 5e-7 * (double)n);
    cudaFreeAsync(scratch, s);
    if (h_passes) *h_passes = count;
    return rc;
}

int psx_fill(float* d_x, size_t n, float value, psx_stream_t stream)
{
    clear_error();
    if (!d_x && n) {
        set_error("fill: null pointer");
        return PSX_ERR_INVALID;
    }
    return launch_fill(d_x, n, value, cs(stream));
}

int psx_convert_u8_f32(const uint8_t* d_in, float* d_out, size_t n, psx_stream_t stream)
{
    clear_error();
    if (!d_in || !d_out) {
        set_error("convert: null pointer");
        return PSX_ERR_INVALID;
    }
    if (!n) return PSX_OK;
    k_convert<uint8_t><<<grid_for(n, 256), 256, 0, cs(stream)>>>(d_in, d_out, n);
    return launch_status("convert kernel");
}

int psx_convert_i8_f32(const int8_t* d_in, float* d_out, size_t n, psx_stream_t stream)
{
    clear_error();
    if (!d_in || !d_out) {
        set_error("convert: null pointer");
        return PSX_ERR_INVALID;
    }
    if (!n) return PSX_OK;
    k_convert<int8_t><<<grid_for(n, 256), 256, 0, cs(stream)>>>(d_in, d_out, n);
    return launch_status("convert kernel");
}

int psx_harmonic_sum(const float* d_in, float* const* h_out_ptrs, size_t n, int nharms,
                     psx_stream_t stream)
{
    clear_error();
    if (!d_in || n == 0 || n > 0x7fffffffu || nharms < 0 || nharms > 5 ||
        (nharms && !h_out_ptrs)) {
        set_error("harmonic_sum: bad arguments (nharms must be 0..5)");
        return PSX_ERR_INVALID;
    }
    if (nharms == 0) return PSX_OK;
    FoldPtrs o{};
    for (int h = 0; h < nharms; ++h) {
        if (!h_out_ptrs[h]) {
            set_error("harmonic_sum: null output %d", h);
            return PSX_ERR_INVALID;
        }
        o.p[h] = h_out_ptrs[h];
    }
    k_harmonic_sum<<<grid_for(n, 256), 256, 0, cs(stream)>>>(d_in, o, (unsigned)n, nharms);
    return launch_status("harmonic sum kernel");
}

int psx_find_peaks(const float* d_spec, int n, int start, float thresh, int* d_idx,
                   float* d_val, int cap, int* h_count, psx_stream_t stream)
{
    clear_error();
    if (!d_spec || !h_count || (cap > 0 && (!d_idx || !d_val))) {
        set_error("find_peaks: bad arguments");
        return PSX_ERR_INVALID;
    }
    if (start < 0) start = 0;
    *h_count = 0;
    if (n <= start) return PSX_OK;
    cudaStream_t s = cs(stream);
    const int ntiles = (n - start + kCompactTile - 1) / kCompactTile;
    int* scratch = nullptr;
    PSX_CUDA(cudaMallocAsync((void**)&scratch, sizeof(int) * (ntiles + 1), s));
    k_compact_count<<<ntiles, 256, 0, s>>>(d_spec, start, n, thresh, scratch);
    k_compact_scan<<<1, 32, 0, s>>>(scratch, ntiles, scratch + ntiles);
    k_compact_write<<<ntiles, 256, 0, s>>>(d_spec, start, n, thresh, scratch, d_idx, d_val, cap);
    int rc = launch_status("compaction kernels");
    int total = 0;
    if (rc == PSX_OK)
        rc = cuda_status(cudaMemcpyAsync(&total, scratch + ntiles, sizeof(int),
                                         cudaMemcpyDeviceToHost, s), "find_peaks copy");
    cudaFreeAsync(scratch, s);
    if (rc == PSX_OK) rc = cuda_status(cudaStreamSynchronize(s), "find_peaks");
    if (rc != PSX_OK) return rc;
    *h_count = total;
    if (total > cap) {
        set_error("find_peaks: %d values above threshold, buffer holds %d", total, cap);
        return PSX_ERR_OVERFLOW;
    }
    return PSX_OK;
}

}  // extern "C"

// ------------------------------------------------- peak finding, no allocation
// psx_find_peaks_noalloc runs the three compaction kernels of psx_find_peaks
// with their per-tile counts in a fixed device array instead of memory from
// cudaMallocAsync.  It serves callers that may not allocate device memory
// while they search: hosts that have handed the whole of a GPU's memory to
// their own pool or to another framework, hosts that forbid allocation
// after start-up so that memory use cannot grow during a run, and code
// running where an allocation could block or fail at a bad moment.
//
// The array g_peak_tile_scratch is compiled into this library: every GPU
// that loads the library holds its 256 KiB (+ 4 bytes) until the process
// exits.  It has room for kNoAllocMaxTiles tile counts plus the total, so a
// call may scan at most kNoAllocMaxTiles * kCompactTile = 2^28 bins
// (n - start).  All calls on a device share the one array and it keeps the
// last call's contents; nothing in it needs to start at zero, because
// k_compact_count writes every tile count a call uses before k_compact_scan
// reads it.  Calls whose GPU work overlaps (other streams, other host
// threads) race on the array and give wrong results.
namespace psx {
namespace {

constexpr int kNoAllocMaxTiles = 65536;
constexpr long long kNoAllocMaxBins = (long long)kNoAllocMaxTiles * kCompactTile;
constexpr int kNoAllocMaxDevices = 64;

// Device-side storage.  In host code this name is only a handle for the
// runtime's symbol lookup, never a pointer that can be dereferenced or
// passed to a kernel.
static __device__ __align__(256) int g_peak_tile_scratch[kNoAllocMaxTiles + 1];

std::mutex g_peak_scratch_mu;
int* g_peak_scratch_addr[kNoAllocMaxDevices] = {nullptr};

// The device address of g_peak_tile_scratch on the current device, looked
// up once per device (the first call on each device does it, with that
// device current) and cached.
int peak_scratch_address(int** out)
{
    int dev = -1;
    PSX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error("find_peaks_noalloc: device ordinal %d outside 0..%d", dev,
                  kNoAllocMaxDevices - 1);
        return PSX_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_peak_scratch_mu);
    if (!g_peak_scratch_addr[dev]) {
        void* p = nullptr;
        PSX_CUDA(cudaGetSymbolAddress(&p, g_peak_tile_scratch));
        if (!p) {
            set_error("find_peaks_noalloc: no device address for the scratch array");
            return PSX_ERR_CUDA;
        }
        g_peak_scratch_addr[dev] = static_cast<int*>(p);
    }
    *out = g_peak_scratch_addr[dev];
    return PSX_OK;
}

}  // namespace
}  // namespace psx

extern "C" int psx_find_peaks_noalloc(const float* d_spec, int n, int start, float thresh,
                                      int* d_idx, float* d_val, int cap, int* h_count,
                                      psx_stream_t stream)
{
    clear_error();
    if (!d_spec || !h_count || (cap > 0 && (!d_idx || !d_val))) {
        set_error("find_peaks_noalloc: bad arguments");
        return PSX_ERR_INVALID;
    }
    if (start < 0) start = 0;
    *h_count = 0;
    if (n <= start) return PSX_OK;
    if ((long long)n - start > kNoAllocMaxBins) {
        set_error("find_peaks_noalloc: %lld bins to scan, the static scratch holds at most %lld "
                  "(use psx_find_peaks)", (long long)n - start, kNoAllocMaxBins);
        return PSX_ERR_INVALID;
    }
    int* scratch = nullptr;
    int rc = peak_scratch_address(&scratch);
    if (rc != PSX_OK) return rc;
    cudaStream_t s = cs(stream);
    const int ntiles = (n - start + kCompactTile - 1) / kCompactTile;
    k_compact_count<<<ntiles, 256, 0, s>>>(d_spec, start, n, thresh, scratch);
    k_compact_scan<<<1, 32, 0, s>>>(scratch, ntiles, scratch + ntiles);
    k_compact_write<<<ntiles, 256, 0, s>>>(d_spec, start, n, thresh, scratch, d_idx, d_val, cap);
    rc = launch_status("compaction kernels");
    int total = 0;
    if (rc == PSX_OK)
        rc = cuda_status(cudaMemcpyAsync(&total, scratch + ntiles, sizeof(int),
                                         cudaMemcpyDeviceToHost, s), "find_peaks_noalloc copy");
    if (rc == PSX_OK) rc = cuda_status(cudaStreamSynchronize(s), "find_peaks_noalloc");
    if (rc != PSX_OK) return rc;
    *h_count = total;
    if (total > cap) {
        set_error("find_peaks_noalloc: %d values above threshold, buffer holds %d", total, cap);
        return PSX_ERR_OVERFLOW;
    }
    return PSX_OK;
}
