// psx_fft4.cu -- the batched search's forward transform, written for
// sm_100a: per acceleration trial the complex DFT of length M = N/2 of
// z[m] = x'[2m] + i x'[2m+1] (x' the resampled series) as a four-step
// transform M = R * C (R = 1024, or 768 for lengths 3 * 2^k) in two passes
// over HBM, then the real-spectrum
// unpack fused with interbinning and normalisation.
//
// It replaces, on the batched path, the reference's resample kernel
// (src/kernels.cu:364-380), its cuFFT R2C call (include/transforms/
// ffter.hpp:23-53) and the spectrum forming and normalising kernels
// (src/kernels.cu:238-259, :496-507) with three launches:
//   pass 1 (k_fft4_cols): CTA = 8 columns c of the R x C matrix
//     z[r * C + c], 512 threads; each thread gathers 16 rows of its column
//     straight from the dereddened series through the resample index (FP64,
//     the same device function the resample kernel reads through), then Stockham
//     stages of radix 16, 16 and 4 in registers with two exchanges through
//     shared memory, the four-step twiddle W_M^(c k1), then y[k1 * C + c];
//   pass 2 (k_fft4_rows): CTA = one row k1 (or 256/(C/16) rows) of y,
//     radix-16 Stockham stages (one radix 2/4/8 stage where C is not a
//     power of 16) through padded shared memory, written in natural order
//     as zt[k1 * C + k2] = Z[k1 + R k2];
//   unpack (k_unpack_form_norm_t): a CTA stages a 32-row x 32-column tile of
//     zt and the tile of its mirror bins through shared memory with
//     coalesced asynchronous copies; then lanes take consecutive k1 (30
//     output lanes and two helpers per warp), so the neighbour bin k-1 each
//     interbinned value needs is the previous lane's, and the mirror bin
//     M-k the next lane's.
// All twiddles come from tables rounded once from double precision (pass 1
// takes some as the product of two entries, or of one entry and an exact
// multiple of pi/8, to read fewer of them).
#include <cuda_runtime.h>
#include <cmath>
#include <utility>
#include <vector>
#include "psx_common.cuh"
#include "psx_device.cuh"
#include "psx_fft4.cuh"

namespace psx {

namespace {


// cos(k pi / 16), k = 0..8
__host__ __device__ constexpr float cos_pi16(int k)
{
    return k == 0   ? 1.0f
           : k == 1 ? 0.980785280403230449126f
           : k == 2 ? 0.923879532511286756128f
           : k == 3 ? 0.831469612302545237079f
           : k == 4 ? 0.707106781186547524401f
           : k == 5 ? 0.555570233019602224743f
           : k == 6 ? 0.382683432365089771728f
           : k == 7 ? 0.195090322016128267848f
                    : 0.0f;
}

// cos and sin of 2 pi m / 32
__host__ __device__ constexpr float cos32(int m)
{
    m &= 31;
    return m <= 8 ? cos_pi16(m) : m <= 16 ? -cos_pi16(16 - m) : m <= 24 ? -cos_pi16(m - 16)
                                                                        : cos_pi16(32 - m);
}
__host__ __device__ constexpr float sin32(int m) { return cos32(8 - m); }

__device__ __forceinline__ float2 cmul(float2 a, float2 w)
{
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// a * W_L^k with W_L = exp(-2 pi i / L), L <= 32 (k, L constants after
// unrolling; the quarter turns are swaps and sign changes)
__device__ __forceinline__ float2 twiddle(float2 a, int k, int L)
{
    const int m = (k * (32 / L)) & 31;
    if (m == 0) return a;
    if (m == 8) return make_float2(a.y, -a.x);
    if (m == 16) return make_float2(-a.x, -a.y);
    if (m == 24) return make_float2(-a.y, a.x);
    return cmul(a, make_float2(cos32(m), -sin32(m)));
}

__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x / 2); }

template <int I, int BITS>
struct BitRev {
    static constexpr int value = ((I & 1) << (BITS - 1)) | BitRev<(I >> 1), BITS - 1>::value;
};
template <int I>
struct BitRev<I, 0> {
    static constexpr int value = 0;
};

// One radix-2 decimation-in-frequency stage over blocks of 2*SPAN, then
// the next one.
template <int L, int SPAN>
__device__ __forceinline__ void dif_stage(float2 (&v)[L])
{
#pragma unroll
    for (int b = 0; b < L; b += 2 * SPAN) {
#pragma unroll
        for (int k = 0; k < SPAN; ++k) {
            const float2 a = v[b + k], c = v[b + k + SPAN];
            v[b + k] = make_float2(a.x + c.x, a.y + c.y);
            v[b + k + SPAN] = twiddle(make_float2(a.x - c.x, a.y - c.y), k, 2 * SPAN);
        }
    }
    if constexpr (SPAN > 1) dif_stage<L, SPAN / 2>(v);
}

template <int L, int... I>
__device__ __forceinline__ void unscramble(float2 (&v)[L], std::integer_sequence<int, I...>)
{
    constexpr int LOG = ilog2(L);
    const float2 t[L] = {v[BitRev<I, LOG>::value]...};
    ((v[I] = t[I]), ...);
}

// Forward DFT of length L (2..32) in registers, natural order in and out:
// radix-2 decimation in frequency, then the bit reversal as a renaming.
template <int L>
__device__ __forceinline__ void dft(float2 (&v)[L])
{
    dif_stage<L, L / 2>(v);
    unscramble(v, std::make_integer_sequence<int, L>{});
}

// Forward DFT of length 3: with W = exp(-2 pi i / 3) = -1/2 - i s, s = sqrt(3)/2,
// X1,2 = a - (b + c)/2 -/+ i s (b - c).
__device__ __forceinline__ void dft3(float2& a, float2& b, float2& c)
{
    constexpr float s3 = 0.866025403784438646763723f;
    const float2 t1 = make_float2(b.x + c.x, b.y + c.y);
    const float2 t2 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
    const float2 d = make_float2(b.x - c.x, b.y - c.y);
    const float2 m = make_float2(s3 * d.y, -s3 * d.x);
    a = make_float2(a.x + t1.x, a.y + t1.y);
    b = make_float2(t2.x + m.x, t2.y + m.y);
    c = make_float2(t2.x - m.x, t2.y - m.y);
}

// ------------------------------------------------------------- pass 1
// Column shape of pass 1 for column length R: W columns per CTA, J = R/16
// radix-16 butterflies per column in the first two stages, TPC threads per
// column (J, at least 64), a last stage of radix R3 = R/256 with U = 256/TPC
// butterflies per thread; 16 elements (12 for R = 768) per thread.  W is at
// least 4 so that every row a CTA reads or writes is one whole 32-byte
// sector (the series of a long segment does not stay in L2): 512 threads
// and 64 KB of shared memory for R <= 2048, 1024 threads and 128 KB (one
// CTA per SM) for R = 4096.
template <int R>
struct ColShape {
    static constexpr int W = R >= 2048 ? 4 : 8;
    static constexpr int J = R / 16;
    static constexpr int TPC = J < 64 ? 64 : J;
    static constexpr int R3 = R / 256;
    static constexpr int U = 256 / TPC;
    static constexpr int THREADS = W * TPC;
    static constexpr size_t SMEM = (size_t)R * W * sizeof(float2);
};

// Shared layout [e][col], e the row index 0..R-1; a row of W columns spans
// 2W of the 32 banks.  XOR-ing the low bits of e with bits 4.. of e (16/W
// row groups) spreads the rows a warp touches at once (32/W consecutive t)
// over all the banks in every exchange below: two wavefronts per 64-bit
// access, the minimum.
template <int W>
__device__ __forceinline__ unsigned swz_a(unsigned e)
{
    return e ^ ((e >> 4) & (16u / W - 1u));
}

// Column length R = 768 (stages of radix 16, 16, 3, for transform lengths
// 3 * 2^k), 1024 (16, 16, 4), 2048 (16, 16, 8) or 4096 (16, 16, 16).
// DUMP: write the gathered pairs z[e C + c] (the resampled series as it is
// read, interleaved) to y instead of transforming them (the debug tap).
template <int R, bool DUMP>
__global__ void __launch_bounds__(ColShape<R>::THREADS, 1024 / ColShape<R>::THREADS)
    k_fft4_cols(const float* __restrict__ x, unsigned long long n, const double* __restrict__ ktab,
                const float2* __restrict__ tab, unsigned offA2, unsigned offA3, unsigned offQ,
                unsigned offP, unsigned C, float2* __restrict__ y, size_t ypitch,
                const unsigned* __restrict__ trow, size_t xpitch)
{
    using S = ColShape<R>;
    // trials of several series (trow: trial -> row of x, rows xpitch apart)
    if (trow) x += (size_t)trow[blockIdx.y] * xpitch;
    static_assert(R == 768 || R == 1024 || R == 2048 || R == 4096, "column length");
    static_assert((S::THREADS == 512 || S::THREADS == 1024) && S::U * S::R3 <= 16,
                  "column shape");
    constexpr int W = S::W, J = S::J, TPC = S::TPC, R3 = S::R3, U = S::U;
    extern __shared__ float2 sm_a[];
    const unsigned col = threadIdx.x % W, t = threadIdx.x / W;  // t in [0, TPC)
    const unsigned c = blockIdx.x * W + col;
    const double k = ktab[blockIdx.y], size = (double)n;
    // Table entries of the four-step twiddle (last step below), loaded first
    // so that their L2 latency passes under the three stages; for R = 4096
    // (one stage-3 butterfly per thread, fifteen entries W_M^(TPC c U q))
    // those are loaded where they are used instead.
    constexpr bool EARLY = U > 1;
    const float2 wt = __ldg(tab + offQ + (size_t)t * C + c);
    float2 pu[U], pq[R3];
    if constexpr (EARLY) {
        // P = W_M^(TPC c): P^u and (P^U)^q as products of two entries
        pu[1] = __ldg(tab + offP + (size_t)C + c);
        pq[1] = __ldg(tab + offP + (size_t)U * C + c);
#pragma unroll
        for (int u = 2; u < U; ++u) pu[u] = cmul(pu[u / 2], pu[u - u / 2]);
#pragma unroll
        for (int q = 2; q < R3; ++q) pq[q] = cmul(pq[q / 2], pq[q - q / 2]);
    }
    float2 v[16];
    // stage 1 (radix 16, span 1): rows e = t + J q of column c, where
    // z[e C + c] = (x'[2m], x'[2m+1]); out[16 t + q]
    if (J == TPC || t < (unsigned)J) {  // every thread unless R = 768
        const double i_first = 2.0 * ((double)t * (double)C + (double)c);
        const double i_step = 2.0 * J * (double)C;
        const unsigned n32 = (unsigned)n;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const double i0 = i_first + (double)q * i_step;  // exact: integers < 2^28
            v[q].x = resampleII_read(x, i0, k, size, n32);
            v[q].y = resampleII_read(x, i0 + 1.0, k, size, n32);
        }
        if constexpr (DUMP) {
            float2* yo = y + (size_t)blockIdx.y * ypitch;
#pragma unroll
            for (int q = 0; q < 16; ++q) yo[(size_t)(t + J * q) * C + c] = v[q];
        } else {
            dft<16>(v);
#pragma unroll
            for (int q = 0; q < 16; ++q) sm_a[swz_a<W>(16 * t + q) * W + col] = v[q];
        }
    }
    if constexpr (DUMP) return;
    __syncthreads();
    // stage 2 (radix 16, span 16): in[t + J q] * W_256^((t mod 16) q),
    // out[(t / 16) 256 + t mod 16 + 16 q]
    if (J == TPC || t < (unsigned)J) {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = sm_a[swz_a<W>(t + J * q) * W + col];
    }
    __syncthreads();
    if (J == TPC || t < (unsigned)J) {
        // W_256^(m q) = W_256^(m (q mod 4)) W_256^(4 m (q div 4)): six table
        // entries instead of fifteen
        const float2* a2 = tab + offA2 + (t & 15);
        const float2 one = make_float2(1.0f, 0.0f);
        const float2 lo[4] = {one, __ldg(a2 + 16), __ldg(a2 + 32), __ldg(a2 + 48)};
        const float2 hi[4] = {one, __ldg(a2 + 64), __ldg(a2 + 128), __ldg(a2 + 192)};
#pragma unroll
        for (int q = 1; q < 16; ++q) {
            const int ql = q & 3, qh = q >> 2;
            v[q] = cmul(v[q], !qh ? lo[ql] : !ql ? hi[qh] : cmul(lo[ql], hi[qh]));
        }
        dft<16>(v);
        const unsigned base2 = (t >> 4) * 256 + (t & 15);
#pragma unroll
        for (int q = 0; q < 16; ++q) sm_a[swz_a<W>(base2 + 16 * q) * W + col] = v[q];
    }
    __syncthreads();
    // stage 3 (radix R3, span 256): butterflies j = t + TPC u, in[j + 256 q]
    // * W_R^(j q), out[j + 256 q] = row k1 = t + TPC (u + U q)
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < R3; ++q)
            v[R3 * u + q] = sm_a[swz_a<W>(t + TPC * u + 256 * q) * W + col];
    // With R = 16 TPC, W_R^(j q) = W_R^(t q) W_16^(u q): R3 - 1 table entries
    // and exact multiples of pi/8 instead of U (R3 - 1) entries (R = 768
    // reads them all).
    constexpr bool SPLIT3 = R == 16 * TPC;
    float2 w3[R3];
    if constexpr (SPLIT3)
#pragma unroll
        for (int q = 1; q < R3; ++q) w3[q] = __ldg(tab + offA3 + q * 256 + t);
#pragma unroll
    for (int u = 0; u < U; ++u) {
        float2 b[R3];
#pragma unroll
        for (int q = 0; q < R3; ++q) {
            if (!q)
                b[q] = v[R3 * u];
            else if constexpr (SPLIT3)
                b[q] = twiddle(cmul(v[R3 * u + q], w3[q]), u * q, 16);
            else
                b[q] = cmul(v[R3 * u + q], __ldg(tab + offA3 + q * 256 + t + TPC * u));
        }
        if constexpr (R3 == 3) {
            dft3(b[0], b[1], b[2]);
        } else {
            dft<R3>(b);
        }
#pragma unroll
        for (int q = 0; q < R3; ++q) v[R3 * u + q] = b[q];
    }
    // four-step twiddle W_M^(c k1), k1 = t + TPC w (w = u + U q):
    // W_M^(c t) * W_M^(TPC c U q) * W_M^(TPC c u), from the entries of
    // W_M^(c t), W_M^(TPC c) and W_M^(TPC c U) instead of U R3 (R = 4096:
    // W_M^(c t) and the fifteen W_M^(TPC c q))
    float2* yo = y + (size_t)blockIdx.y * ypitch;
#pragma unroll
    for (int q = 0; q < R3; ++q) {
        const float2 wq =
            q ? cmul(wt, EARLY ? pq[q] : __ldg(tab + offP + (size_t)(U * q) * C + c)) : wt;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const unsigned w = u + U * q;
            const float2 tw = u ? cmul(wq, pu[u]) : wq;
            yo[(size_t)(t + TPC * w) * C + c] = cmul(v[R3 * u + q], tw);
        }
    }
}

// ------------------------------------------------------------- pass 2
__device__ __forceinline__ unsigned pad16(unsigned a) { return a + (a >> 4); }

template <int LOGC>
struct RowShape {
    static constexpr int C = 1 << LOGC, T = C / 16, RPC = T >= 256 ? 1 : 256 / T;
    static constexpr int REM = LOGC % 4, R1 = REM ? (1 << REM) : 16;
    static constexpr int NST = LOGC / 4 + (REM ? 1 : 0);
    static constexpr int THREADS = T * RPC;
    static constexpr size_t SMEM = (size_t)RPC * (C + C / 16) * sizeof(float2);
    // twiddle table offset of the last stage (stage s >= 1 holds R_s * NS_s)
    static constexpr int OFF_LAST = NST == 2 ? 0 : NST == 3 ? 16 * R1 : 16 * R1 + 256 * R1;
};

// One Stockham stage of radix R and span NS in place in shared memory over
// a row of C elements, T = C/16 threads: thread t takes the butterflies
// j = t + u T (u < 16/R).
template <int R, int NS, int C>
__device__ __forceinline__ void row_stage(float2* s, unsigned t, const float2* __restrict__ tw)
{
    constexpr int T = C / 16, G = 16 / R;
    float2 v[16];
#pragma unroll
    for (int u = 0; u < G; ++u)
#pragma unroll
        for (int q = 0; q < R; ++q) v[u * R + q] = s[pad16(t + u * T + q * (C / R))];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < G; ++u) {
        const unsigned jb = t + u * T, m = jb % NS;
        float2 w[R];
        if constexpr (R == 16) {
            // W^(m q) = W^(m (q mod 4)) W^(4 m (q div 4)): six entries, not 15
            const float2 one = make_float2(1.0f, 0.0f);
            const float2 lo[4] = {one, __ldg(tw + NS + m), __ldg(tw + 2 * NS + m),
                                  __ldg(tw + 3 * NS + m)};
            const float2 hi[4] = {one, __ldg(tw + 4 * NS + m), __ldg(tw + 8 * NS + m),
                                  __ldg(tw + 12 * NS + m)};
            w[0] = v[u * R];
#pragma unroll
            for (int q = 1; q < 16; ++q) {
                const int ql = q & 3, qh = q >> 2;
                w[q] = cmul(v[u * R + q], !qh ? lo[ql] : !ql ? hi[qh] : cmul(lo[ql], hi[qh]));
            }
        } else {
#pragma unroll
            for (int q = 0; q < R; ++q)
                w[q] = q ? cmul(v[u * R + q], __ldg(tw + q * NS + m)) : v[u * R];
        }
        dft<R>(w);
        const unsigned base = (jb / NS) * NS * R + m;
#pragma unroll
        for (int q = 0; q < R; ++q) s[pad16(base + q * NS)] = w[q];
    }
    __syncthreads();
}

template <int LOGC>
__global__ void __launch_bounds__(RowShape<LOGC>::THREADS, 1024 / RowShape<LOGC>::THREADS)
    k_fft4_rows(const float2* __restrict__ y, size_t ypitch, float2* __restrict__ zt,
                size_t zpitch, const float2* __restrict__ tw)
{
    using S = RowShape<LOGC>;
    constexpr int C = S::C, T = S::T;
    extern __shared__ float2 sm_b[];
    const unsigned lr = threadIdx.x / T, t = threadIdx.x % T;
    const unsigned row = blockIdx.x * S::RPC + lr;
    float2* s = sm_b + lr * (C + C / 16);
    const float2* yr = y + (size_t)blockIdx.y * ypitch + (size_t)row * C;
    float2 v[16];
    // stage 0: radix 16, span 1, from the row in HBM
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = yr[t + q * T];
    dft<16>(v);
#pragma unroll
    for (int q = 0; q < 16; ++q) s[pad16(t * 16 + q)] = v[q];
    __syncthreads();
    if constexpr (S::NST >= 3) row_stage<S::R1, 16, C>(s, t, tw);
    if constexpr (S::NST >= 4) row_stage<16, 16 * S::R1, C>(s, t, tw + 16 * S::R1);
    // last stage: radix 16, span C/16, natural order straight to HBM
    constexpr int NSL = C / 16;
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = s[pad16(t + q * T)];
    {
        // W_C^(t q) from six entries, as in row_stage
        const float2* tl = tw + S::OFF_LAST + t;
        const float2 one = make_float2(1.0f, 0.0f);
        const float2 lo[4] = {one, __ldg(tl + NSL), __ldg(tl + 2 * NSL), __ldg(tl + 3 * NSL)};
        const float2 hi[4] = {one, __ldg(tl + 4 * NSL), __ldg(tl + 8 * NSL), __ldg(tl + 12 * NSL)};
#pragma unroll
        for (int q = 1; q < 16; ++q) {
            const int ql = q & 3, qh = q >> 2;
            v[q] = cmul(v[q], !qh ? lo[ql] : !ql ? hi[qh] : cmul(lo[ql], hi[qh]));
        }
    }
    dft<16>(v);
    float2* zr = zt + (size_t)blockIdx.y * zpitch + (size_t)row * C;
#pragma unroll
    for (int q = 0; q < 16; ++q) zr[t + q * T] = v[q];
}

// ------------------------------------------------------------- unpack
template <unsigned R>
__device__ __forceinline__ float2 zt_at(const float2* __restrict__ z, unsigned C, unsigned idx)
{
    return z[(size_t)(idx % R) * C + (idx / R)];
}

// 2 X[j] and 2 X[M-j] of the real series from Z[j] = a and Z[M-j] = w,
// with (cs, sn) = (cos, sin)(pi j / M) (the split step of a real transform
// computed as a half-length complex one).  The factor 2 is kept: the
// interbinned amplitude of 2X is exactly twice that of X (a power-of-two
// scale commutes with rounding, square root included), and normalising
// with twice the mean and twice the deviation gives exactly the same value,
// so the four halvings per pair are not needed.
__device__ __forceinline__ void unpack_one(float2 a, float2 w, float cs, float sn, float2& lo,
                                           float2& hi)
{
    const float ar = a.x + w.x, ai = a.y - w.y, br = a.x - w.x, bi = a.y + w.y;
    const float u = cs * bi - sn * br, v = sn * bi + cs * br;
    lo = make_float2(ar + u, ai - v);
    hi = make_float2(ar - u, -ai - v);
}

// 8-byte asynchronous copy from global to shared memory: no register holds
// the element while it is in flight.
__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Grid (ceil(R/30) * C/64, trials), 256 threads, R the row count of the
// four-step split (1024 or 768).  CTA (wk, g): rows
// k1 = 30 wk - 1 + r, r < 32 ("virtual" rows -1 and >= R continue into
// the neighbouring columns), columns k2 = 32 g .. 32 g + 31 < C/2: the bins
// j = k1 + R k2 < M/2 and their mirrors M - j.  Both 32 x 32 tiles are
// copied coalesced (a warp reads 32 consecutive columns of a row) into
// padded shared memory by asynchronous copies; warp w then takes columns 32 g + 4 w .. + 3 with
// lane = r, and lanes 1..30 write bin j (interbinned with lane-1's X[j-1])
// and bin M-j (with lane+1's X[M-j-1]); bin M/2 comes from thread 0 of
// block 0.  The split-step rotation (cos, sin)(pi j / M) is the product of
// tabulated (cos, sin)(pi k1 / M) (k1 = -1 .. 1055, rv[k1 + 1]) and
// (cos, sin)(pi k2 / C) (rk[k2]).
template <unsigned R>
__global__ void __launch_bounds__(256, 8)  // 8 CTAs per SM: 32 registers
    k_unpack_form_norm_t(const float2* __restrict__ zt, size_t zpitch, unsigned C,
                         float* __restrict__ p, size_t ppitch,
                         const float2* __restrict__ rv, const float2* __restrict__ rk,
                         const float* __restrict__ stat, const unsigned* __restrict__ trow)
{
    __shared__ float2 lo_t[32][33], mi_t[32][33];
    // trials of several series: trial blockIdx.y's statistics at row trow[]
    if (trow) stat += 8u * trow[blockIdx.y];
    const unsigned M = R * C;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned gblocks = C / 64;
    const unsigned wk = blockIdx.x / gblocks;
    const unsigned k2a = (blockIdx.x % gblocks) * 32;
    const int v0 = (int)(30 * wk) - 1;
    const float2* z = zt + (size_t)blockIdx.y * zpitch;
    float* o = p + (size_t)blockIdx.y * ppitch;
    if (v0 >= 1 && v0 + 31 < (int)R) {  // every row a real row: direct addresses
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const unsigned r = warp + 8 * e;  // tile row; lane = tile column
            const unsigned v = (unsigned)v0 + r;
            cp_async8(&lo_t[r][lane], z + (size_t)v * C + k2a + lane);
            cp_async8(&mi_t[r][lane], z + (size_t)(R - v) * C + (C - 1 - k2a - lane));
        }
        cp_async_commit();
        cp_async_wait<0>();
    } else
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const unsigned r = warp + 8 * e;  // tile row; lane = tile column
        const long long j = (long long)(v0 + (int)r) + (long long)R * (k2a + lane);
        float2 a = make_float2(0.f, 0.f), w = a;  // X[-1] := 0
        if (j >= 0) {
            const unsigned jj = (unsigned)j;
            a = zt_at<R>(z, C, jj);
            w = zt_at<R>(z, C, jj ? M - jj : 0u);
        }
        lo_t[r][lane] = a;
        mi_t[r][lane] = w;
    }
    __syncthreads();
    const int k1v = v0 + (int)lane;
    const float2 tv = __ldg(rv + (k1v + 1));
    const float meanN = 2.0f * stat[3], stdN = 2.0f * stat[4];  // of 2X (exact)
    const bool out = lane >= 1 && lane <= 30 && k1v < (int)R;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const unsigned cc = 4 * warp + t, k2 = k2a + cc;
        const float2 tk = __ldg(rk + k2);
        const float cs = tv.x * tk.x - tv.y * tk.y, sn = tv.y * tk.x + tv.x * tk.y;
        float2 lo, hi;
        unpack_one(lo_t[lane][cc], mi_t[lane][cc], cs, sn, lo, hi);
        if (k1v < 0 && k2 == 0) lo = hi = make_float2(0.f, 0.f);
        const float plx = __shfl_up_sync(0xffffffffu, lo.x, 1);
        const float ply = __shfl_up_sync(0xffffffffu, lo.y, 1);
        const float nhx = __shfl_down_sync(0xffffffffu, hi.x, 1);
        const float nhy = __shfl_down_sync(0xffffffffu, hi.y, 1);
        if (out) {
            const unsigned j = (unsigned)k1v + R * k2;
            o[j] = normalise(interbin(lo.x, lo.y, plx, ply), meanN, stdN);
            o[M - j] = normalise(interbin(hi.x, hi.y, nhx, nhy), meanN, stdN);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // bin M/2 with bin M/2 - 1
        // (cos, sin)(pi/2) = (0, 1); (cos, sin)(pi/2 - pi/M) = (sin, cos)(pi/M)
        const unsigned jh = M / 2;
        const float2 r1 = __ldg(rv + 2);  // (cos, sin)(pi / M)
        float2 x0, x1, unused;
        unpack_one(zt_at<R>(z, C, jh), zt_at<R>(z, C, M - jh), 0.0f, 1.0f, x0, unused);
        unpack_one(zt_at<R>(z, C, jh - 1), zt_at<R>(z, C, M - jh + 1), r1.y, r1.x, x1, unused);
        o[jh] = normalise(interbin(x0.x, x0.y, x1.x, x1.y), meanN, stdN);
    }
}

template <int LOGC>
int configure_rows()
{
    using S = RowShape<LOGC>;
    if (S::SMEM <= 48 * 1024) return PSX_OK;
    return cuda_status(cudaFuncSetAttribute(k_fft4_rows<LOGC>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)S::SMEM),
                       "fft4 row pass attribute");
}

template <int LOGC>
int launch_rows(unsigned nrows, const float2* y, size_t ypitch, float2* zt, size_t zpitch,
                const float2* tw, int ntrials, cudaStream_t s)
{
    using S = RowShape<LOGC>;
    dim3 grid(nrows / S::RPC, (unsigned)ntrials);
    k_fft4_rows<LOGC><<<grid, S::THREADS, S::SMEM, s>>>(y, ypitch, zt, zpitch, tw);
    return launch_status("fft4 row pass");
}

// Stages of the row pass: (radix, span) for stage 1 .. NST-1 (stage 0 has
// no twiddles), as RowShape lays them out.
void row_stages(int logc, std::vector<std::pair<int, int>>& out)
{
    const int rem = logc % 4, r1 = rem ? (1 << rem) : 16;
    const int nst = logc / 4 + (rem ? 1 : 0);
    out.clear();
    int ns = 16;
    for (int s = 1; s < nst; ++s) {
        const int r = s == 1 ? r1 : 16;
        out.emplace_back(r, ns);
        ns *= r;
    }
}

template <int R>
int configure_cols()
{
    using S = ColShape<R>;
    // (the default shared/L1 split: measured on B200, forcing the largest
    // shared carve-out slowed the gather of pass 1 and the twiddle reads of
    // pass 2, both served from L1)
    return cuda_status(cudaFuncSetAttribute(k_fft4_cols<R, false>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)S::SMEM),
                       "fft4 column pass attribute");
}

}  // namespace

template <int R, bool DUMP>
void Fft4Plan::launch_cols(const Fft4Plan& f, const float* series, const double* ktab,
                           int ntrials, float2* y, size_t ypitch, cudaStream_t s,
                           const unsigned* trow, size_t xpitch)
{
    using S = ColShape<R>;
    dim3 ga(f.C / S::W, (unsigned)ntrials);
    k_fft4_cols<R, DUMP><<<ga, S::THREADS, DUMP ? 0 : S::SMEM, s>>>(
        series, (unsigned long long)f.n, ktab, f.d_tab, f.offA2, f.offA3, f.offQ, f.offP, f.C, y,
        ypitch, trow, xpitch);
}

bool Fft4Plan::supported(size_t n)
{
    auto pow2 = [](size_t v) { return v && (v & (v - 1)) == 0; };
    if (pow2(n)) return n >= (size_t(1) << 19) && n <= (size_t(1) << 27);
    return n % 3 == 0 && pow2(n / 3) && n / 3 >= (size_t(1) << 17) && n / 3 <= (size_t(1) << 23);
}

// Rows of the four-step split: 768 for 3 * 2^k, else 1024 up to M = 2^24
// (N = 2^25), 2048 at M = 2^25 and 4096 at M = 2^26, so that the row length
// C = M / R never exceeds 2^14 (one CTA's shared memory).
unsigned Fft4Plan::rows_for(size_t n)
{
    const size_t m = n / 2;
    if (n % 3 == 0) return 768u;
    return m <= (size_t(1) << 24) ? 1024u : m == (size_t(1) << 25) ? 2048u : 4096u;
}

// Threads per column of pass 1 (the range of t in the four-step twiddle).
static unsigned cols_tpc(unsigned r) { return r / 16 < 64 ? 64u : r / 16; }

size_t Fft4Plan::table_floats2(size_t n)
{
    const unsigned r = rows_for(n), c = (unsigned)(n / 2 / r);
    int lc = 0;
    while ((1u << lc) < c) ++lc;
    std::vector<std::pair<int, int>> st;
    row_stages(lc, st);
    size_t rows = 0;
    for (auto& e : st) rows += (size_t)e.first * e.second;
    return 256 + (size_t)(r / 256) * 256 + (size_t)cols_tpc(r) * c + 16 * (size_t)c +
           (r + 33) + c / 2 + rows;
}

void Fft4Plan::destroy()
{
    if (d_tab) cudaFree(d_tab);
    d_tab = nullptr;
    tab_len = 0;
    n = 0;
}

int Fft4Plan::create(size_t n_)
{
    destroy();
    if (!supported(n_)) {
        set_error("fft4: unsupported length %zu (2^19 .. 2^27 or 3 * 2^17 .. 3 * 2^23)", n_);
        return PSX_ERR_INVALID;
    }
    const unsigned long long M = n_ / 2;
    const unsigned Rn = rows_for(n_);
    const unsigned R3 = Rn / 256;
    const unsigned Cn = (unsigned)(M / Rn);
    const unsigned tpc = cols_tpc(Rn);
    const double two_pi = 6.283185307179586476925286766559;
    // W_L^e = exp(-2 pi i e / L), rounded once from double
    auto W = [&](unsigned long long e, unsigned long long L) {
        e %= L;
        const double a = two_pi * (double)e / (double)L;
        return make_float2((float)std::cos(a), (float)-std::sin(a));
    };
    std::vector<float2> h;
    h.reserve(table_floats2(n_));
    offA2 = 0;  // [q * 16 + m] = W_256^(m q)
    for (unsigned q = 0; q < 16; ++q)
        for (unsigned m = 0; m < 16; ++m) h.push_back(W((unsigned long long)m * q, 256));
    offA3 = (unsigned)h.size();  // [q * 256 + j] = W_R^(j q)
    for (unsigned q = 0; q < R3; ++q)
        for (unsigned j = 0; j < 256; ++j) h.push_back(W((unsigned long long)j * q, Rn));
    offQ = (unsigned)h.size();  // [t * C + c] = W_M^(c t), t < threads per column
    for (unsigned t = 0; t < tpc; ++t)
        for (unsigned c = 0; c < Cn; ++c) h.push_back(W((unsigned long long)c * t, M));
    offP = (unsigned)h.size();  // [w * C + c] = W_M^(tpc c w), w < 16
    for (unsigned w = 0; w < 16; ++w)
        for (unsigned c = 0; c < Cn; ++c) h.push_back(W((unsigned long long)tpc * c * w, M));
    // unpack rotations (cos, sin)(pi k1 / M), k1 = -1 .. R + 31, and (pi k2 / C)
    const double pi = two_pi / 2;
    offRv = (unsigned)h.size();
    for (int k1 = -1; k1 <= (int)Rn + 31; ++k1)
        h.push_back(make_float2((float)std::cos(pi * k1 / (double)M),
                                (float)std::sin(pi * k1 / (double)M)));
    offRk = (unsigned)h.size();
    for (unsigned k2 = 0; k2 < Cn / 2; ++k2)
        h.push_back(make_float2((float)std::cos(pi * k2 / Cn), (float)std::sin(pi * k2 / Cn)));
    offB = (unsigned)h.size();  // row-pass stages: [q * NS + m] = W_(R NS)^(q m)
    int lc = 0;
    while ((1u << lc) < Cn) ++lc;
    std::vector<std::pair<int, int>> stages;
    row_stages(lc, stages);
    for (auto& rs : stages)
        for (int q = 0; q < rs.first; ++q)
            for (int m = 0; m < rs.second; ++m)
                h.push_back(W((unsigned long long)q * m, (unsigned long long)rs.first * rs.second));
    PSX_CUDA(cudaMalloc(&d_tab, sizeof(float2) * h.size()));
    tab_len = h.size();
    PSX_CUDA(cudaMemcpy(d_tab, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice));
    n = n_;
    C = Cn;
    R = Rn;
    logc = lc;
    switch (R) {
    case 768: PSX_TRY(configure_cols<768>()); break;
    case 1024: PSX_TRY(configure_cols<1024>()); break;
    case 2048: PSX_TRY(configure_cols<2048>()); break;
    default: PSX_TRY(configure_cols<4096>()); break;
    }

    switch (logc) {
    case 8: return configure_rows<8>();
    case 9: return configure_rows<9>();
    case 10: return configure_rows<10>();
    case 11: return configure_rows<11>();
    case 12: return configure_rows<12>();
    case 13: return configure_rows<13>();
    case 14: return configure_rows<14>();
    default: break;
    }
    set_error("fft4: row length 2^%d out of range", logc);
    return PSX_ERR_INVALID;
}

int Fft4Plan::exec(const float* series, const double* ktab, int ntrials, float2* y,
                   size_t ypitch, float2* zt, size_t zpitch, cudaStream_t s) const
{
    PSX_TRY(exec_cols(series, ktab, ntrials, y, ypitch, s, nullptr, 0));
    return exec_rows(y, ypitch, ntrials, zt, zpitch, s);
}

int Fft4Plan::exec_cols(const float* series, const double* ktab, int ntrials, float2* y,
                        size_t ypitch, cudaStream_t s, const unsigned* trow,
                        size_t xpitch) const
{
    if (!d_tab || !series || !ktab || !y || ntrials <= 0 || ntrials > 65535 || ypitch < n / 2 ||
        (trow && xpitch < n)) {
        set_error("fft4: bad arguments");
        return PSX_ERR_INVALID;
    }
    const unsigned* tr = trow;
    const size_t xp = xpitch;
    switch (R) {
    case 768: launch_cols<768, false>(*this, series, ktab, ntrials, y, ypitch, s, tr, xp); break;
    case 1024: launch_cols<1024, false>(*this, series, ktab, ntrials, y, ypitch, s, tr, xp); break;
    case 2048: launch_cols<2048, false>(*this, series, ktab, ntrials, y, ypitch, s, tr, xp); break;
    default: launch_cols<4096, false>(*this, series, ktab, ntrials, y, ypitch, s, tr, xp); break;
    }
    return launch_status("fft4 column pass");
}

int Fft4Plan::dump_gather(const float* series, const double* ktab, float* out,
                          cudaStream_t s) const
{
    if (!d_tab || !series || !ktab || !out) {
        set_error("fft4 dump: bad arguments");
        return PSX_ERR_INVALID;
    }
    float2* o = reinterpret_cast<float2*>(out);
    switch (R) {
    case 768: launch_cols<768, true>(*this, series, ktab, 1, o, n / 2, s, nullptr, 0); break;
    case 1024: launch_cols<1024, true>(*this, series, ktab, 1, o, n / 2, s, nullptr, 0); break;
    case 2048: launch_cols<2048, true>(*this, series, ktab, 1, o, n / 2, s, nullptr, 0); break;
    default: launch_cols<4096, true>(*this, series, ktab, 1, o, n / 2, s, nullptr, 0); break;
    }
    return launch_status("fft4 gather dump");
}

int Fft4Plan::exec_rows(const float2* y, size_t ypitch, int ntrials, float2* zt, size_t zpitch,
                        cudaStream_t s) const
{
    if (!d_tab || !y || !zt || ntrials <= 0 || ntrials > 65535 || ypitch < n / 2 ||
        zpitch < n / 2) {
        set_error("fft4: bad arguments");
        return PSX_ERR_INVALID;
    }
    const float2* tw = d_tab + offB;
    switch (logc) {
    case 8: return launch_rows<8>(R, y, ypitch, zt, zpitch, tw, ntrials, s);
    case 9: return launch_rows<9>(R, y, ypitch, zt, zpitch, tw, ntrials, s);
    case 10: return launch_rows<10>(R, y, ypitch, zt, zpitch, tw, ntrials, s);
    case 11: return launch_rows<11>(R, y, ypitch, zt, zpitch, tw, ntrials, s);
    case 12: return launch_rows<12>(R, y, ypitch, zt, zpitch, tw, ntrials, s);
    case 13: return launch_rows<13>(R, y, ypitch, zt, zpitch, tw, ntrials, s);
    case 14: return launch_rows<14>(R, y, ypitch, zt, zpitch, tw, ntrials, s);
    default: break;
    }
    set_error("fft4: row length 2^%d out of range", logc);
    return PSX_ERR_INVALID;
}

int Fft4Plan::form(const float2* zt, size_t zpitch, int ntrials, float* p, size_t ppitch,
                   const float* stat, cudaStream_t s, const unsigned* trow) const
{
    if (!d_tab || !zt || !p || !stat || ntrials <= 0 || ntrials > 65535 || zpitch < n / 2 ||
        ppitch < n / 2 + 1) {
        set_error("fft4 form: bad arguments");
        return PSX_ERR_INVALID;
    }
    const unsigned nck = (R + 29) / 30;
    dim3 grid(nck * (C / 64), (unsigned)ntrials);
    const float2* rv = d_tab + offRv;
    const float2* rk = d_tab + offRk;
    switch (R) {
    case 768: k_unpack_form_norm_t<768><<<grid, 256, 0, s>>>(zt, zpitch, C, p, ppitch, rv, rk, stat, trow); break;
    case 1024: k_unpack_form_norm_t<1024><<<grid, 256, 0, s>>>(zt, zpitch, C, p, ppitch, rv, rk, stat, trow); break;
    case 2048: k_unpack_form_norm_t<2048><<<grid, 256, 0, s>>>(zt, zpitch, C, p, ppitch, rv, rk, stat, trow); break;
    default: k_unpack_form_norm_t<4096><<<grid, 256, 0, s>>>(zt, zpitch, C, p, ppitch, rv, rk, stat, trow); break;
    }
    return launch_status("fft4 unpack kernel");
}

}  // namespace psx
