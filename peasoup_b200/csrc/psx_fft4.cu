// psx_fft4.cu -- the batched search's forward transform, written for
// sm_100a: per acceleration trial the complex DFT of length M = N/2 of
// z[m] = x'[2m] + i x'[2m+1] (x' the resampled series) as a four-step
// transform M = 1024 * C in two passes over HBM, then the real-spectrum
// unpack fused with interbinning and normalisation.
//
// It replaces, on the batched path, the reference's resample kernel
// (src/kernels.cu:364-380), its cuFFT R2C call (include/transforms/
// ffter.hpp:23-53) and the spectrum forming and normalising kernels
// (src/kernels.cu:238-259, :496-507) with three launches:
//   pass 1 (k_fft4_cols): CTA = 8 columns c of the 1024 x C matrix
//     z[r * C + c]; each thread gathers 32 rows of its column straight from
//     the dereddened series through the resample index (FP64, the same
//     device function the resample kernel uses), a radix-32 Stockham stage
//     in registers, one exchange through shared memory, the second radix-32
//     stage, the four-step twiddle W_M^(c k1), then y[k1 * C + c];
//   pass 2 (k_fft4_rows): CTA = one row k1 (or 256/(C/16) rows) of y,
//     radix-16 Stockham stages (one radix 2/4/8 stage where C is not a
//     power of 16) through padded shared memory, written in natural order
//     as zt[k1 * C + k2] = Z[k1 + 1024 k2];
//   unpack (k_unpack_form_norm_t): lanes take consecutive k1 (30 output
//     lanes and two helpers per warp), so the neighbour bin k-1 each
//     interbinned value needs is the previous lane's, and the mirror bin
//     M-k the next lane's.
// All twiddles come from tables rounded once from double precision.
#include <cuda_runtime.h>
#include <cmath>
#include <utility>
#include <vector>
#include "psx_common.cuh"
#include "psx_device.cuh"
#include "psx_fft4.cuh"

namespace psx {

namespace {

constexpr int kColsW = 8;  // columns per pass-1 CTA

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

// ------------------------------------------------------------- pass 1
// Shared layout [e][col], e the row index 0..1023; with 8 columns a row is
// 64 bytes, and flipping bit 0 of e by bit 5 puts the four rows a warp
// touches at once two in each half of the banks.
template <int W>
__device__ __forceinline__ unsigned swz_a(unsigned e)
{
    return W == 16 ? e : (e ^ ((e >> 5) & 1u));
}

template <int W>
__global__ void __launch_bounds__(W * 32, 2)
    k_fft4_cols(const float* __restrict__ x, unsigned long long n, const double* __restrict__ ktab,
                const float2* __restrict__ tab, unsigned offA, unsigned offQ, unsigned offP,
                unsigned C, float2* __restrict__ y, size_t ypitch)
{
    extern __shared__ float2 sm_a[];
    const unsigned col = threadIdx.x % W, j = threadIdx.x / W;  // j in [0, 32)
    const unsigned c = blockIdx.x * W + col;
    const double k = ktab[blockIdx.y], size = (double)n;
    float2 v[32];
    // rows e = j + 32 q of column c: z[e C + c] = (x'[2m], x'[2m+1])
#pragma unroll
    for (int q = 0; q < 32; ++q) {
        const unsigned long long i0 = 2ull * ((unsigned long long)(j + 32 * q) * C + c);
        v[q].x = gather_at(x, resampleII_index(i0, k, size), n);
        v[q].y = gather_at(x, resampleII_index(i0 + 1, k, size), n);
    }
    // Stockham radix 32, span 1: out[32 j + q]
    dft<32>(v);
#pragma unroll
    for (int q = 0; q < 32; ++q) sm_a[swz_a<W>(32 * j + q) * W + col] = v[q];
    __syncthreads();
    // span 32: in[j + 32 q] * W_1024^(j q), out[j + 32 q] = row k1 of the column DFT
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = sm_a[swz_a<W>(j + 32 * q) * W + col];
#pragma unroll
    for (int q = 1; q < 32; ++q) v[q] = cmul(v[q], __ldg(tab + offA + q * 32 + j));
    dft<32>(v);
    // four-step twiddle W_M^(c k1), k1 = j + 32 q: W_M^(c j) * W_M^(32 c q)
    const float2 wq = __ldg(tab + offQ + (size_t)j * C + c);
    float2* yo = y + (size_t)blockIdx.y * ypitch;
#pragma unroll
    for (int q = 0; q < 32; ++q) {
        const float2 w = q ? cmul(wq, __ldg(tab + offP + (size_t)q * C + c)) : wq;
        yo[(size_t)(j + 32 * q) * C + c] = cmul(v[q], w);
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
#pragma unroll
        for (int q = 0; q < R; ++q)
            w[q] = q ? cmul(v[u * R + q], __ldg(tw + q * NS + m)) : v[u * R];
        dft<R>(w);
        const unsigned base = (jb / NS) * NS * R + m;
#pragma unroll
        for (int q = 0; q < R; ++q) s[pad16(base + q * NS)] = w[q];
    }
    __syncthreads();
}

template <int LOGC>
__global__ void __launch_bounds__(RowShape<LOGC>::THREADS)
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
#pragma unroll
    for (int q = 1; q < 16; ++q) v[q] = cmul(v[q], __ldg(tw + S::OFF_LAST + q * NSL + t));
    dft<16>(v);
    float2* zr = zt + (size_t)blockIdx.y * zpitch + (size_t)row * C;
#pragma unroll
    for (int q = 0; q < 16; ++q) zr[t + q * T] = v[q];
}

// ------------------------------------------------------------- unpack
struct UnpackSteps {
    float2 w[4];
};

__device__ __forceinline__ float2 zt_at(const float2* __restrict__ z, unsigned C, unsigned idx)
{
    return z[(size_t)(idx & (kFft4Rows - 1)) * C + (idx >> 10)];
}

// X[j] and X[M-j] of the real series from Z[j] = a and Z[M-j] = w, with
// (cs, sn) = (cos, sin)(pi j / M) (the split step of a real transform
// computed as a half-length complex one).
__device__ __forceinline__ void unpack_one(float2 a, float2 w, float cs, float sn, float2& lo,
                                           float2& hi)
{
    const float ar = a.x + w.x, ai = a.y - w.y, br = a.x - w.x, bi = a.y + w.y;
    const float u = cs * bi - sn * br, v = sn * bi + cs * br;
    lo = make_float2(0.5f * (ar + u), 0.5f * (ai - v));
    hi = make_float2(0.5f * (ar - u), 0.5f * (-ai - v));
}

// Grid (ceil(1024/30) * C/64, trials), 256 threads.  Warp (wk, g): lanes
// take rows k1 = 30 wk - 1 + lane ("virtual" rows -1 and >= 1024 continue
// into the neighbouring columns), columns k2 = 4g .. 4g+3 < C/2, i.e. the
// bins j = k1 + 1024 k2 < M/2 and their mirrors M - j.  Lanes 1..30 write
// bin j (interbinned with lane-1's X[j-1]) and bin M-j (with lane+1's
// X[M-j-1]); bin M/2 comes from thread 0 of block 0.
__global__ void __launch_bounds__(256)
    k_unpack_form_norm_t(const float2* __restrict__ zt, size_t zpitch, unsigned C,
                         float* __restrict__ p, size_t ppitch, float inv_m, UnpackSteps st,
                         const float* __restrict__ stat)
{
    constexpr unsigned R = kFft4Rows;
    const unsigned M = R * C;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned gblocks = C / 64;
    const unsigned wk = blockIdx.x / gblocks;
    const unsigned g = (blockIdx.x % gblocks) * 8 + warp;
    const int k1v = (int)(30 * wk + lane) - 1;
    const unsigned k20 = 4 * g;
    const float2* z = zt + (size_t)blockIdx.y * zpitch;
    float* o = p + (size_t)blockIdx.y * ppitch;
    float2 a[4], w[4];
    if (k1v >= 1 && k1v < (int)R) {
        const float4* r4 = reinterpret_cast<const float4*>(z + (size_t)k1v * C + k20);
        const float4 a01 = r4[0], a23 = r4[1];
        // Z[M - j] = zt[(R - k1)][C - 1 - k2]: the group C-4-k20 .. C-1-k20, reversed
        const float4* m4 =
            reinterpret_cast<const float4*>(z + (size_t)(R - k1v) * C + (C - 4 - k20));
        const float4 m01 = m4[0], m23 = m4[1];
        a[0] = make_float2(a01.x, a01.y);
        a[1] = make_float2(a01.z, a01.w);
        a[2] = make_float2(a23.x, a23.y);
        a[3] = make_float2(a23.z, a23.w);
        w[3] = make_float2(m01.x, m01.y);
        w[2] = make_float2(m01.z, m01.w);
        w[1] = make_float2(m23.x, m23.y);
        w[0] = make_float2(m23.z, m23.w);
    } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const long long j = (long long)k1v + (long long)R * (k20 + t);
            if (j < 0) {
                a[t] = w[t] = make_float2(0.f, 0.f);  // X[-1] := 0
            } else {
                const unsigned jj = (unsigned)j;
                a[t] = zt_at(z, C, jj);
                w[t] = zt_at(z, C, jj ? M - jj : 0u);
            }
        }
    }
    float s0, c0;
    sincospif((float)((long long)k1v + (long long)R * k20) * inv_m, &s0, &c0);
    float2 lo[4], hi[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const float2 d = st.w[t];  // angle of column k20 + t = angle(k20) + pi t / C
        const float cs = t ? c0 * d.x - s0 * d.y : c0, sn = t ? s0 * d.x + c0 * d.y : s0;
        unpack_one(a[t], w[t], cs, sn, lo[t], hi[t]);
    }
    const float meanN = stat[3], stdN = stat[4];
    const bool out = lane >= 1 && lane <= 30 && k1v < (int)R;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const float plx = __shfl_up_sync(0xffffffffu, lo[t].x, 1);
        const float ply = __shfl_up_sync(0xffffffffu, lo[t].y, 1);
        const float nhx = __shfl_down_sync(0xffffffffu, hi[t].x, 1);
        const float nhy = __shfl_down_sync(0xffffffffu, hi[t].y, 1);
        if (out) {
            const unsigned j = (unsigned)k1v + R * (k20 + t);
            o[j] = normalise(interbin(lo[t].x, lo[t].y, plx, ply), meanN, stdN);
            o[M - j] = normalise(interbin(hi[t].x, hi[t].y, nhx, nhy), meanN, stdN);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // bin M/2 with bin M/2 - 1
        const unsigned jh = M / 2;
        float2 x0, x1, unused;
        float s, c;
        sincospif((float)jh * inv_m, &s, &c);
        unpack_one(zt_at(z, C, jh), zt_at(z, C, M - jh), c, s, x0, unused);
        sincospif((float)(jh - 1) * inv_m, &s, &c);
        unpack_one(zt_at(z, C, jh - 1), zt_at(z, C, M - jh + 1), c, s, x1, unused);
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
int launch_rows(const float2* y, size_t ypitch, float2* zt, size_t zpitch, const float2* tw,
                int ntrials, cudaStream_t s)
{
    using S = RowShape<LOGC>;
    dim3 grid(kFft4Rows / S::RPC, (unsigned)ntrials);
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

}  // namespace

bool Fft4Plan::supported(size_t n)
{
    return n >= (size_t(1) << 19) && n <= (size_t(1) << 25) && (n & (n - 1)) == 0;
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
        set_error("fft4: unsupported length %zu (powers of two 2^19 .. 2^25)", n_);
        return PSX_ERR_INVALID;
    }
    const unsigned long long M = n_ / 2;
    const unsigned Cn = (unsigned)(M / kFft4Rows);
    const double two_pi = 6.283185307179586476925286766559;
    // W_L^e = exp(-2 pi i e / L), rounded once from double
    auto W = [&](unsigned long long e, unsigned long long L) {
        e %= L;
        const double a = two_pi * (double)e / (double)L;
        return make_float2((float)std::cos(a), (float)-std::sin(a));
    };
    std::vector<float2> h;
    h.reserve(1024 + 66 * (size_t)Cn);
    offA = 0;  // [q * 32 + j] = W_1024^(j q)
    for (unsigned q = 0; q < 32; ++q)
        for (unsigned j = 0; j < 32; ++j) h.push_back(W((unsigned long long)j * q, 1024));
    offQ = (unsigned)h.size();  // [j * C + c] = W_M^(c j)
    for (unsigned j = 0; j < 32; ++j)
        for (unsigned c = 0; c < Cn; ++c) h.push_back(W((unsigned long long)c * j, M));
    offP = (unsigned)h.size();  // [q * C + c] = W_M^(32 c q)
    for (unsigned q = 0; q < 32; ++q)
        for (unsigned c = 0; c < Cn; ++c) h.push_back(W(32ull * c * q, M));
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
    const double pi = two_pi / 2;
    for (int t = 0; t < 4; ++t)
        steps[t] = make_float2((float)std::cos(pi * t / Cn), (float)std::sin(pi * t / Cn));
    n = n_;
    C = Cn;
    logc = lc;
    PSX_TRY(cuda_status(cudaFuncSetAttribute(k_fft4_cols<kColsW>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(kFft4Rows * kColsW * sizeof(float2))),
                        "fft4 column pass attribute"));
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
    if (!d_tab || !series || !ktab || !y || !zt || ntrials <= 0 || ntrials > 65535 ||
        ypitch < n / 2 || zpitch < n / 2) {
        set_error("fft4: bad arguments");
        return PSX_ERR_INVALID;
    }
    dim3 ga(C / kColsW, (unsigned)ntrials);
    k_fft4_cols<kColsW><<<ga, kColsW * 32, kFft4Rows * kColsW * sizeof(float2), s>>>(
        series, (unsigned long long)n, ktab, d_tab, offA, offQ, offP, C, y, ypitch);
    PSX_TRY(launch_status("fft4 column pass"));
    const float2* tw = d_tab + offB;
    switch (logc) {
    case 8: return launch_rows<8>(y, ypitch, zt, zpitch, tw, ntrials, s);
    case 9: return launch_rows<9>(y, ypitch, zt, zpitch, tw, ntrials, s);
    case 10: return launch_rows<10>(y, ypitch, zt, zpitch, tw, ntrials, s);
    case 11: return launch_rows<11>(y, ypitch, zt, zpitch, tw, ntrials, s);
    case 12: return launch_rows<12>(y, ypitch, zt, zpitch, tw, ntrials, s);
    case 13: return launch_rows<13>(y, ypitch, zt, zpitch, tw, ntrials, s);
    case 14: return launch_rows<14>(y, ypitch, zt, zpitch, tw, ntrials, s);
    default: break;
    }
    set_error("fft4: row length 2^%d out of range", logc);
    return PSX_ERR_INVALID;
}

int Fft4Plan::form(const float2* zt, size_t zpitch, int ntrials, float* p, size_t ppitch,
                   const float* stat, cudaStream_t s) const
{
    if (!d_tab || !zt || !p || !stat || ntrials <= 0 || ntrials > 65535 || zpitch < n / 2 ||
        ppitch < n / 2 + 1) {
        set_error("fft4 form: bad arguments");
        return PSX_ERR_INVALID;
    }
    UnpackSteps st;
    for (int t = 0; t < 4; ++t) st.w[t] = steps[t];
    const unsigned nck = (kFft4Rows + 29) / 30;
    dim3 grid(nck * (C / 64), (unsigned)ntrials);
    const float inv_m = 1.0f / (float)(n / 2);
    k_unpack_form_norm_t<<<grid, 256, 0, s>>>(zt, zpitch, C, p, ppitch, inv_m, st, stat);
    return launch_status("fft4 unpack kernel");
}

}  // namespace psx
