// psx_dedisp.cu -- direct incoherent dedispersion of SIGPROC sample rows
// into device-resident series: the producer of the search's input.
//
// The reference calls the external dedisp library through Dedisperser
// (include/transforms/dedisperser.hpp:13-188) and copies every dedispersed
// series back to the host, from where each Worker copies one series at a
// time to the device again (src/pipeline_multi.cu:474-505, 166-170).  Here
// the sample rows are unpacked once into a channel-major layout in HBM and
// the dedispersed block is written where the search reads it.
//
// Arithmetic (the published direct algorithm; dedisp itself is absent):
//   delay_c  = 4.15e3/tsamp * (f_c^-2 - fch1^-2)   samples per unit DM
//   D(d, c)  = round-half-even(float(dm_d * delay_c))
//   sum[d,t] = sum over live channels of x_c[t + D(d, c)]  (exact integer)
//   out[d,t] = sum, or (sum - nchans*m/2) * 1/(m*sqrt(nchans)) + 1/2.
//
// Layout.  cm[c][t]: one row of `pitch` samples (u8 for 1..8-bit input, u16
// for 16-bit) per channel, so that every (channel, time window) a CTA needs
// is one contiguous run.  A CTA owns 8 DM trials (one per warp) and 512
// output samples; per channel it stages the window the 8 trials need,
// [t0 + min D, t0 + 512 + max D), with cp.async in double-buffered chunks of
// channels, then each lane adds 16 outputs per channel from shared memory:
// two aligned 32-bit loads, one funnel shift, and (8-bit samples) two byte
// permutes into packed 16-bit accumulators.  Consecutive CTAs take the same
// time tile for successive DM blocks, so the window is read from HBM once
// and from L2 after that.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "psx_common.cuh"

namespace psx {
namespace {

constexpr int kDdThreads = 256;
constexpr int kDdWarps = 8;    // DM trials per CTA
constexpr int kDdTile8 = 1024; // output samples per CTA, 1..8-bit samples
constexpr int kDdTile16 = 512; // output samples per CTA, 16-bit samples
inline int dd_tile(int elem) { return elem == 1 ? kDdTile8 : kDdTile16; }
constexpr int kUpRows = 64;    // unpack tile: samples
constexpr int kUpChans = 64;   // unpack tile: channels
constexpr float kDmConst = 4.15e3f;

template <int NBITS> struct Sample { using T = uint8_t; };
template <> struct Sample<16> { using T = uint16_t; };

// Channel c of a SIGPROC row: below 8 bits the first channel sits in the
// least significant bits of its byte; 16-bit samples are little-endian.
template <int NBITS>
__device__ __forceinline__ unsigned sigproc_value(const uint8_t* row, int c)
{
    if constexpr (NBITS == 8) {
        return row[c];
    } else if constexpr (NBITS == 16) {
        return (unsigned)row[2 * c] | ((unsigned)row[2 * c + 1] << 8);
    } else {
        unsigned bit = (unsigned)c * NBITS;
        return (row[bit >> 3] >> (bit & 7)) & ((1u << NBITS) - 1u);
    }
}

// Rows [r0, r0 + nrows) of the packed input (rows[0] is row r0) become
// columns of cm; columns [r0 + nrows, r0 + ncols) are zeroed.  One CTA per
// 64 samples x 64 channels, transposed through shared memory; every store
// is 16 bytes.  r0 and ncols' rounding to 64 stay inside the pitch.
template <int NBITS>
__global__ void __launch_bounds__(256) k_unpack_chanmajor(
    const uint8_t* __restrict__ rows, size_t row_bytes, size_t nrows, size_t r0, size_t ncols,
    int nchans, typename Sample<NBITS>::T* __restrict__ cm, size_t pitch, int vec)
{
    using T = typename Sample<NBITS>::T;
    constexpr int kPad = 16 / (int)sizeof(T) / 4;  // row stride 68 B (u8) or 132 B (u16)
    constexpr int kStride = kUpRows + kPad;
    __shared__ __align__(16) T tile[kUpChans * kStride];
    const size_t col0 = (size_t)blockIdx.x * kUpRows;
    const int c0 = blockIdx.y * kUpChans;
    if (vec) {
        // 32-bit loads: a row's 64 channels are 2*NBITS words (rows 4-byte aligned)
        constexpr int kWords = 2 * NBITS;
        constexpr int kPerWord = 32 / NBITS;
        const size_t seg = (size_t)c0 * NBITS / 8;
        for (int i = threadIdx.x; i < kUpRows * kWords; i += blockDim.x) {
            int r = i / kWords, q = i % kWords;
            size_t rr = col0 + r;
            size_t byte = seg + 4 * (size_t)q;
            uint32_t w = 0;
            if (rr < nrows && byte < row_bytes)
                w = *reinterpret_cast<const uint32_t*>(rows + rr * row_bytes + byte);
#pragma unroll
            for (int k = 0; k < kPerWord; ++k) {
                unsigned v;
                if constexpr (NBITS == 16) v = (w >> (16 * k)) & 0xffffu;
                else v = (w >> (k * NBITS)) & ((1u << NBITS) - 1u);
                tile[(q * kPerWord + k) * kStride + r] = (T)v;
            }
        }
    } else {
        for (int i = threadIdx.x; i < kUpRows * kUpChans; i += blockDim.x) {
            int r = i / kUpChans, c = i % kUpChans;
            size_t rr = col0 + r;
            unsigned v = 0;
            if (rr < nrows && c0 + c < nchans) v = sigproc_value<NBITS>(rows + rr * row_bytes, c0 + c);
            tile[c * kStride + r] = (T)v;
        }
    }
    __syncthreads();
    constexpr int kVec = 16 / (int)sizeof(T);           // samples per 16-byte store
    constexpr int kPer = kUpRows / kVec;                // stores per channel
    for (int i = threadIdx.x; i < kUpChans * kPer; i += blockDim.x) {
        int c = i / kPer, q = i % kPer;
        if (c0 + c >= nchans || col0 + (size_t)q * kVec >= ncols) continue;
        const uint32_t* src = reinterpret_cast<const uint32_t*>(tile + c * kStride + q * kVec);
        uint4 w = make_uint4(src[0], src[1], src[2], src[3]);
        *reinterpret_cast<uint4*>(cm + (size_t)(c0 + c) * pitch + r0 + col0 + (size_t)q * kVec) = w;
    }
}

struct DedispArgs {
    const void* cm;
    size_t pitch;           // samples per channel row of cm
    const int* chan;        // [nlive] channel row of each live channel
    const int* lo;          // [ngroups * nlive] window start after t0 (samples)
    const int* off;         // [ndm_pad * nlive] D(d, c) - lo(group of d, c)
    int nlive, ndm, nblk, cc, lwin, group;
    float* out;
    size_t out_pitch, nout;
    float mid, scale;
    int raw;
    int p8, p16;            // channels a byte / a 16-bit sum holds at the input's largest value
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ uint32_t lds32(uint32_t addr)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];\n" : "=r"(v) : "r"(addr));
    return v;
}
template <int OFF>
__device__ __forceinline__ uint32_t lds32o(uint32_t addr)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1+%2];\n" : "=r"(v) : "r"(addr), "n"(OFF));
    return v;
}

__device__ __forceinline__ float map_sum(unsigned s, float mid, float scale, int raw)
{
    float v = (float)s;
    if (!raw) v = __fadd_rn(__fmul_rn(__fsub_rn(v, mid), scale), 0.5f);
    return v;
}

template <typename T, bool FLUSH, bool SMALL>
__global__ void __launch_bounds__(kDdThreads) k_dedisperse(DedispArgs a)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int blk = blockIdx.x % a.nblk;
    constexpr int kTile = sizeof(T) == 1 ? kDdTile8 : kDdTile16;
    const size_t t0 = (size_t)(blockIdx.x / a.nblk) * kTile;
    const int d = blk * kDdWarps + warp;
    const int nwin = kDdWarps / a.group;
    const int gw = warp / a.group;
    const int gbase = blk * kDdWarps / a.group;
    const int win_bytes = a.lwin * (int)sizeof(T);
    const int stage_bytes = a.cc * nwin * win_bytes;
    int* s_off = reinterpret_cast<int*>(smem + 2 * stage_bytes);  // [2][8][cc]
    const int nq = (a.nlive + a.cc - 1) / a.cc;

    auto load_chunk = [&](int q, int st) {
        for (int w = warp; w < a.cc * nwin; w += kDdWarps) {
            int j = w / nwin, g = w % nwin, i = q * a.cc + j;
            if (i >= a.nlive) continue;
            const uint8_t* src = static_cast<const uint8_t*>(a.cm) +
                ((size_t)a.chan[i] * a.pitch + t0 + a.lo[(size_t)(gbase + g) * a.nlive + i]) * sizeof(T);
            uint8_t* dst = smem + st * stage_bytes + w * win_bytes;
            for (int p = lane; p < win_bytes / 16; p += 32) cp_async16(dst + 16 * p, src + 16 * p);
        }
        for (int k = threadIdx.x; k < kDdWarps * a.cc; k += kDdThreads) {
            int ww = k / a.cc, j = k % a.cc, i = q * a.cc + j, dd = blk * kDdWarps + ww;
            s_off[(st * kDdWarps + ww) * a.cc + j] =
                (i < a.nlive && dd < a.ndm) ? a.off[(size_t)dd * a.nlive + i] : 0;
        }
        cp_async_commit();
    };

    const bool active = d < a.ndm;
    float* out = a.out + (size_t)(active ? d : 0) * a.out_pitch;

    if constexpr (sizeof(T) == 1) {
        // lane: outputs t0 + 4*lane + 128*k + {0..3}, k = 0..7, as packed
        // 16-bit pairs; with more channels than a pair holds (p16: 257 at
        // 8 bits) a pair is flushed into 32-bit sums before it can overflow.
        // SMALL (samples of at most 4 bits): the four bytes of a word are
        // summed as they stand, p8 channels at a time (17 at 4 bits, 85 at
        // 2, 255 at 1), before they are spread into the 16-bit pairs.
        constexpr int kUnits = kDdTile8 / 128;
        uint32_t acc[2 * kUnits];
        uint32_t a8[SMALL ? kUnits : 1];
#pragma unroll
        for (int k = 0; k < (SMALL ? kUnits : 1); ++k) a8[k] = 0;
        int since8 = 0;
        // 32-bit sums behind the packed pairs, in shared memory (touched once
        // per 257 channels): s_full[k * 256 + thread], after the offsets
        uint32_t* s_full = reinterpret_cast<uint32_t*>(
            smem + 2 * stage_bytes + 2 * kDdWarps * a.cc * (int)sizeof(int));
#pragma unroll
        for (int k = 0; k < 2 * kUnits; ++k) acc[k] = 0;
        if constexpr (FLUSH) {
#pragma unroll
            for (int k = 0; k < 4 * kUnits; ++k) s_full[k * kDdThreads + threadIdx.x] = 0;
        }
        int since = 0;
        const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(smem);
        const uint32_t s_offs = s_base + 2u * stage_bytes + (uint32_t)warp * a.cc * 4u;
        const uint32_t wstep = (uint32_t)(nwin * win_bytes);
        load_chunk(0, 0);
        for (int q = 0; q < nq; ++q) {
            if (q + 1 < nq) { load_chunk(q + 1, (q + 1) & 1); cp_async_wait<1>(); }
            else cp_async_wait<0>();
            __syncthreads();
            const int st = q & 1;
            const int nj = min(a.cc, a.nlive - q * a.cc);
            if (active) {
                if constexpr (SMALL) {
                    if (since8 + nj > a.p8) {
#pragma unroll
                        for (int k = 0; k < kUnits; ++k) {
                            acc[2 * k] += __byte_perm(a8[k], 0, 0x4140);
                            acc[2 * k + 1] += __byte_perm(a8[k], 0, 0x4342);
                            a8[k] = 0;
                        }
                        since8 = 0;
                    }
                    since8 += nj;
                }
                if constexpr (FLUSH) {
                    if (since + nj > a.p16) {
                        if constexpr (SMALL) {
#pragma unroll
                            for (int k = 0; k < kUnits; ++k) {
                                acc[2 * k] += __byte_perm(a8[k], 0, 0x4140);
                                acc[2 * k + 1] += __byte_perm(a8[k], 0, 0x4342);
                                a8[k] = 0;
                            }
                            since8 = nj;
                        }
#pragma unroll
                        for (int k = 0; k < 2 * kUnits; ++k) {
                            s_full[(2 * k) * kDdThreads + threadIdx.x] += acc[k] & 0xffffu;
                            s_full[(2 * k + 1) * kDdThreads + threadIdx.x] += acc[k] >> 16;
                            acc[k] = 0;
                        }
                        since = 0;
                    }
                    since += nj;
                }
                uint32_t wa = s_base + (uint32_t)(st * stage_bytes + gw * win_bytes) + 4u * lane;
                const uint32_t oa = s_offs + (uint32_t)st * kDdWarps * a.cc * 4u;
#pragma unroll 2
                for (int j = 0; j < nj; ++j, wa += wstep) {
                    const int o = (int)lds32(oa + 4u * j);
                    const uint32_t ad = wa + (uint32_t)(o & ~3);
                    const uint32_t sh = (uint32_t)(o & 3) << 3;
#define PSX_DD_STEP(k)                                                            \
                    {                                                             \
                        uint32_t v = __funnelshift_r(lds32o<128 * (k)>(ad),       \
                                                     lds32o<128 * (k) + 4>(ad), sh); \
                        if constexpr (SMALL) {                                    \
                            a8[(k)] += v;                                         \
                        } else {                                                  \
                            acc[2 * (k)] += __byte_perm(v, 0, 0x4140);            \
                            acc[2 * (k) + 1] += __byte_perm(v, 0, 0x4342);        \
                        }                                                         \
                    }
                    PSX_DD_STEP(0)
                    PSX_DD_STEP(1)
                    PSX_DD_STEP(2)
                    PSX_DD_STEP(3)
                    PSX_DD_STEP(4)
                    PSX_DD_STEP(5)
                    PSX_DD_STEP(6)
                    PSX_DD_STEP(7)
#undef PSX_DD_STEP
                }
            }
            __syncthreads();
        }
        if (!active) return;
        if constexpr (SMALL) {
#pragma unroll
            for (int k = 0; k < kUnits; ++k) {
                acc[2 * k] += __byte_perm(a8[k], 0, 0x4140);
                acc[2 * k + 1] += __byte_perm(a8[k], 0, 0x4342);
            }
        }
#pragma unroll
        for (int k = 0; k < kUnits; ++k) {
            uint32_t s0 = acc[2 * k] & 0xffffu, s1 = acc[2 * k] >> 16;
            uint32_t s2 = acc[2 * k + 1] & 0xffffu, s3 = acc[2 * k + 1] >> 16;
            if constexpr (FLUSH) {
                s0 += s_full[(4 * k) * kDdThreads + threadIdx.x];
                s1 += s_full[(4 * k + 1) * kDdThreads + threadIdx.x];
                s2 += s_full[(4 * k + 2) * kDdThreads + threadIdx.x];
                s3 += s_full[(4 * k + 3) * kDdThreads + threadIdx.x];
            }
            size_t t = t0 + 4 * lane + 128 * k;
            float4 v = make_float4(map_sum(s0, a.mid, a.scale, a.raw),
                                   map_sum(s1, a.mid, a.scale, a.raw),
                                   map_sum(s2, a.mid, a.scale, a.raw),
                                   map_sum(s3, a.mid, a.scale, a.raw));
            if (t + 3 < a.nout) {
                *reinterpret_cast<float4*>(out + t) = v;
            } else {
                if (t < a.nout) out[t] = v.x;
                if (t + 1 < a.nout) out[t + 1] = v.y;
                if (t + 2 < a.nout) out[t + 2] = v.z;
            }
        }
    } else {
        // 16-bit samples: lane outputs t0 + 2*lane + 64*k + {0, 1}, k = 0..7
        uint32_t full[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        load_chunk(0, 0);
        for (int q = 0; q < nq; ++q) {
            if (q + 1 < nq) { load_chunk(q + 1, (q + 1) & 1); cp_async_wait<1>(); }
            else cp_async_wait<0>();
            __syncthreads();
            const int st = q & 1;
            const int nj = min(a.cc, a.nlive - q * a.cc);
            if (active) {
                const uint8_t* wbase = smem + st * stage_bytes + gw * win_bytes;
                const int* offs = s_off + (st * kDdWarps + warp) * a.cc;
                for (int j = 0; j < nj; ++j) {
                    const uint32_t* w = reinterpret_cast<const uint32_t*>(wbase + j * nwin * win_bytes);
                    const int o = offs[j] + 2 * lane;
                    const int sh = (o & 1) * 16;
                    const int wi = o >> 1;
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        uint32_t v = __funnelshift_r(w[wi + 32 * k], w[wi + 32 * k + 1], sh);
                        full[2 * k] += v & 0xffffu;
                        full[2 * k + 1] += v >> 16;
                    }
                }
            }
            __syncthreads();
        }
        if (!active) return;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            size_t t = t0 + 2 * lane + 64 * k;
            float2 v = make_float2(map_sum(full[2 * k], a.mid, a.scale, a.raw),
                                   map_sum(full[2 * k + 1], a.mid, a.scale, a.raw));
            if (t + 1 < a.nout) *reinterpret_cast<float2*>(out + t) = v;
            else if (t < a.nout) out[t] = v.x;
        }
    }
}

size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

}  // namespace
}  // namespace psx

using namespace psx;

struct psx_dedisp_plan {
    size_t nchans = 0;
    float tsamp = 0, fch1 = 0, foff = 0;
    std::vector<float> delays, dms;
    std::vector<int> live;  // 1 = channel summed
    // derived tables for one sample width (elem bytes), rebuilt when dirty
    bool dirty = true;
    int elem = 0;
    int nlive = 0, ndm_pad = 0, nblk = 0, group = 8, lwin = 0, cc = 0;
    size_t ngroups = 0, max_lo = 0;
    size_t scratch_limit = 4ull << 30;  // bytes of channel-major samples
    size_t flush_bytes = 0;             // shared 32-bit sums above 257 channels
    std::vector<int> h_tab;
    int* d_tab = nullptr;
    size_t tab_cap = 0;
    void* d_cm = nullptr;
    size_t cm_cap = 0;
    uint8_t* d_stage = nullptr;
    size_t stage_cap = 0;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copied[2] = {nullptr, nullptr};
    cudaEvent_t ev_used[2] = {nullptr, nullptr};

    size_t max_delay() const
    {
        if (dms.empty() || nchans == 0) return 0;
        float dm_max = dms[0];
        for (float v : dms) dm_max = std::max(dm_max, v);
        float prod = dm_max * delays[nchans - 1];
        return (size_t)std::floor((double)prod + 0.5);
    }

    // Shift tables and the window shape for `el`-byte samples.
    int build_tables(int el)
    {
        if (!dirty && el == elem) return PSX_OK;
        if (dms.empty()) {
            set_error("psx_dedisp: no DM list set");
            return PSX_ERR_INVALID;
        }
        std::vector<int> chans;
        for (size_t c = 0; c < nchans; ++c)
            if (live[c]) chans.push_back((int)c);
        nlive = (int)chans.size();
        const int ndm = (int)dms.size();
        ndm_pad = (int)round_up((size_t)ndm, kDdWarps);
        nblk = ndm_pad / kDdWarps;
        const int align = 16 / el;  // window starts on 16-byte boundaries
        std::vector<int> shift((size_t)ndm * std::max(nlive, 1));
        for (int d = 0; d < ndm; ++d)
            for (int i = 0; i < nlive; ++i) {
                float p = dms[d] * delays[chans[i]];
                shift[(size_t)d * nlive + i] = (int)std::nearbyint(p);
            }
        // window shape for groups of G trials: lo = min shift aligned down,
        // lwin covers 512 outputs past the largest shift plus the read-ahead
        auto shape = [&](int G, std::vector<int>* lo_out, int* lwin_out, size_t* max_lo_out) {
            size_t ng = (size_t)ndm_pad / G;
            std::vector<int> lo(ng * std::max(nlive, 1), 0);
            int spread = 0;
            size_t mlo = 0;
            for (size_t g = 0; g < ng; ++g)
                for (int i = 0; i < nlive; ++i) {
                    int mn = INT32_MAX, mx = 0;
                    for (int d = (int)g * G; d < std::min(ndm, (int)(g + 1) * G); ++d) {
                        int s = shift[(size_t)d * nlive + i];
                        mn = std::min(mn, s);
                        mx = std::max(mx, s);
                    }
                    if (mn == INT32_MAX) mn = mx = 0;
                    int l = mn / align * align;
                    lo[g * nlive + i] = l;
                    spread = std::max(spread, mx - l);
                    mlo = std::max(mlo, (size_t)l);
                }
            *lwin_out = (int)round_up((size_t)spread + dd_tile(el) + 8, (size_t)align);
            *max_lo_out = mlo;
            if (lo_out) lo_out->swap(lo);
        };
        std::vector<int> lo8, lo1;
        int lwin8 = 0, lwin1 = 0;
        size_t mlo8 = 0, mlo1 = 0;
        shape(8, &lo8, &lwin8, &mlo8);
        shape(1, &lo1, &lwin1, &mlo1);
        group = (lwin8 <= kDdWarps * lwin1) ? 8 : 1;
        std::vector<int>& lo = group == 8 ? lo8 : lo1;
        lwin = group == 8 ? lwin8 : lwin1;
        max_lo = group == 8 ? mlo8 : mlo1;
        ngroups = (size_t)ndm_pad / group;
        const int nwin = kDdWarps / group;
        cc = 0;
        flush_bytes = (el == 1 && nlive > 257) ? 4ull * (kDdTile8 / 32) * kDdThreads : 0;
        // with the flush sums, fewer channels per chunk keep 4 CTAs on an SM
        const size_t cap = flush_bytes ? 56 * 1024 : 96 * 1024;
        for (int c : {16, 8, 4, 2, 1}) {
            size_t bytes = 2ull * c * nwin * lwin * el + 2ull * kDdWarps * c * sizeof(int) +
                           flush_bytes;
            if (bytes <= cap || (c == 1 && bytes <= 200 * 1024)) {
                cc = c;
                break;
            }
        }
        if (cc == 0) {
            set_error("psx_dedisp: DM trials of one block spread over %d samples; "
                      "the shared-memory window does not fit", lwin);
            return PSX_ERR_UNSUPPORTED;
        }
        h_tab.assign((size_t)nlive + ngroups * nlive + (size_t)ndm_pad * nlive, 0);
        std::copy(chans.begin(), chans.end(), h_tab.begin());
        std::copy(lo.begin(), lo.begin() + ngroups * nlive, h_tab.begin() + nlive);
        int* off = h_tab.data() + nlive + ngroups * nlive;
        for (int d = 0; d < ndm; ++d)
            for (int i = 0; i < nlive; ++i)
                off[(size_t)d * nlive + i] =
                    shift[(size_t)d * nlive + i] - lo[(size_t)(d / group) * nlive + i];
        elem = el;
        dirty = true;  // tables must be uploaded
        return PSX_OK;
    }

    size_t smem_bytes() const
    {
        return 2ull * cc * (kDdWarps / group) * lwin * elem + 2ull * kDdWarps * cc * sizeof(int) +
               flush_bytes;
    }

    ~psx_dedisp_plan()
    {
        if (d_tab) cudaFree(d_tab);
        if (d_cm) cudaFree(d_cm);
        if (d_stage) cudaFree(d_stage);
        for (int i = 0; i < 2; ++i) {
            if (ev_copied[i]) cudaEventDestroy(ev_copied[i]);
            if (ev_used[i]) cudaEventDestroy(ev_used[i]);
        }
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }
};

namespace {

int grow(void** p, size_t* cap, size_t need, const char* what)
{
    if (*cap >= need) return PSX_OK;
    if (*p) {
        cudaFree(*p);  // synchronises the device: no launch still reads it
        *p = nullptr;
        *cap = 0;
    }
    cudaError_t e = cudaMalloc(p, need);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error("psx_dedisp: cannot allocate %zu bytes for %s: %s", need, what,
                  cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? PSX_ERR_ALLOC : PSX_ERR_CUDA;
    }
    *cap = need;
    return PSX_OK;
}

int check_input(psx_dedisp_plan* p, size_t nsamps, int nbits, float* d_out, size_t out_pitch,
                size_t* nout)
{
    if (!p) {
        set_error("psx_dedisp: null plan");
        return PSX_ERR_INVALID;
    }
    if (nbits != 1 && nbits != 2 && nbits != 4 && nbits != 8 && nbits != 16) {
        set_error("psx_dedisp: %d-bit samples are not supported (1, 2, 4, 8, 16)", nbits);
        return PSX_ERR_UNSUPPORTED;
    }
    if ((p->nchans * (size_t)nbits) % 8 != 0) {
        set_error("psx_dedisp: a row of %zu %d-bit channels is not whole bytes", p->nchans, nbits);
        return PSX_ERR_INVALID;
    }
    size_t md = p->max_delay();
    if (p->dms.empty() || nsamps <= md) {
        set_error("psx_dedisp: %zu samples do not exceed the maximum delay %zu", nsamps, md);
        return PSX_ERR_INVALID;
    }
    if (!d_out || (reinterpret_cast<uintptr_t>(d_out) & 15) || out_pitch % 4 != 0 ||
        out_pitch < nsamps - md) {
        set_error("psx_dedisp: output must be 16-byte aligned with a pitch (multiple of 4) "
                  "of at least %zu floats", nsamps - md);
        return PSX_ERR_INVALID;
    }
    *nout = nsamps - md;
    return PSX_OK;
}

// Tables uploaded and cm sized.  The outputs are made in gulps of *gulp
// samples (a multiple of the CTA tile) so that cm, *pitch samples per
// channel, stays within the plan's scratch limit; one gulp covers the
// whole series when it fits.
int prepare(psx_dedisp_plan* p, size_t nout, int el, cudaStream_t st, size_t* gulp,
            size_t* pitch)
{
    bool rebuilt = p->dirty || el != p->elem;
    PSX_TRY(p->build_tables(el));
    if (rebuilt) {
        size_t bytes = p->h_tab.size() * sizeof(int);
        PSX_TRY(grow(reinterpret_cast<void**>(&p->d_tab), &p->tab_cap, std::max<size_t>(bytes, 4),
                     "shift tables"));
        PSX_CUDA(cudaMemcpyAsync(p->d_tab, p->h_tab.data(), bytes, cudaMemcpyHostToDevice, st));
        p->dirty = false;
    }
    const size_t tile = dd_tile(el);
    const size_t md = p->max_delay();
    auto pitch_for = [&](size_t g) {
        size_t nt = (g + tile - 1) / tile;
        size_t need = (nt - 1) * tile + p->max_lo + (size_t)p->lwin;
        return round_up(std::max(need, g + md), kUpRows);
    };
    size_t g = round_up(nout, tile);
    const size_t limit = p->scratch_limit / (p->nchans * (size_t)el);
    if (pitch_for(g) > limit) {
        size_t fixed = pitch_for(tile) - tile;
        g = limit > fixed + tile ? (limit - fixed) / tile * tile : tile;
    }
    *gulp = g;
    *pitch = pitch_for(g);
    return grow(&p->d_cm, &p->cm_cap, *pitch * p->nchans * el, "channel-major samples");
}

template <int NBITS>
int launch_unpack(const uint8_t* rows, size_t nrows, size_t r0, size_t ncols, psx_dedisp_plan* p,
                  size_t pitch, cudaStream_t st)
{
    using T = typename Sample<NBITS>::T;
    size_t row_bytes = p->nchans * NBITS / 8;
    dim3 grid((unsigned)((ncols + kUpRows - 1) / kUpRows),
              (unsigned)((p->nchans + kUpChans - 1) / kUpChans));
    // word loads when every row starts 4-byte aligned; channels past the
    // last whole word of a row then read as zero and are never stored
    const int vec = (row_bytes % 4 == 0 && (reinterpret_cast<uintptr_t>(rows) & 3) == 0) ? 1 : 0;
    k_unpack_chanmajor<NBITS><<<grid, 256, 0, st>>>(rows, row_bytes, nrows, r0, ncols,
                                                    (int)p->nchans, static_cast<T*>(p->d_cm), pitch,
                                                    vec);
    return launch_status("k_unpack_chanmajor");
}

int unpack(int nbits, const uint8_t* rows, size_t nrows, size_t r0, size_t ncols,
           psx_dedisp_plan* p, size_t pitch, cudaStream_t st)
{
    switch (nbits) {
        case 1: return launch_unpack<1>(rows, nrows, r0, ncols, p, pitch, st);
        case 2: return launch_unpack<2>(rows, nrows, r0, ncols, p, pitch, st);
        case 4: return launch_unpack<4>(rows, nrows, r0, ncols, p, pitch, st);
        case 8: return launch_unpack<8>(rows, nrows, r0, ncols, p, pitch, st);
        default: return launch_unpack<16>(rows, nrows, r0, ncols, p, pitch, st);
    }
}

int dedisperse(psx_dedisp_plan* p, int nbits, size_t pitch, size_t nout, float* d_out,
               size_t out_pitch, int flags, cudaStream_t st)
{
    DedispArgs a;  // with every channel killed the sums are zero
    a.cm = p->d_cm;
    a.pitch = pitch;
    a.chan = p->d_tab;
    a.lo = p->d_tab + p->nlive;
    a.off = p->d_tab + p->nlive + p->ngroups * p->nlive;
    a.nlive = p->nlive;
    a.ndm = (int)p->dms.size();
    a.nblk = p->nblk;
    a.cc = p->cc;
    a.lwin = p->lwin;
    a.group = p->group;
    a.out = d_out;
    a.out_pitch = out_pitch;
    a.nout = nout;
    unsigned m = (1u << nbits) - 1u;
    a.mid = (float)(0.5 * (double)p->nchans * (double)m);
    a.scale = (float)(1.0 / ((double)m * std::sqrt((double)p->nchans)));
    a.raw = (flags & PSX_DEDISP_RAW) ? 1 : 0;
    a.p8 = (int)(255u / m);
    a.p16 = (int)(65535u / m);
    const size_t tile = dd_tile(nbits == 16 ? 2 : 1);
    size_t ntiles = (nout + tile - 1) / tile;
    size_t nblocks = ntiles * (size_t)p->nblk;
    if (nblocks > 0x7fffffffull) {
        set_error("psx_dedisp: %zu blocks exceed one launch", nblocks);
        return PSX_ERR_UNSUPPORTED;
    }
    size_t smem = p->smem_bytes();
    const unsigned grid = (unsigned)nblocks;
    if (nbits == 16) {
        PSX_CUDA(cudaFuncSetAttribute(k_dedisperse<uint16_t, false, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_dedisperse<uint16_t, false, false><<<grid, kDdThreads, smem, st>>>(a);
    } else {
        // 8 bits and below: the flush and small-sample variants
        const bool flush = p->nlive > a.p16, small = nbits <= 4;
        auto kern = small ? (flush ? k_dedisperse<uint8_t, true, true>
                                   : k_dedisperse<uint8_t, false, true>)
                          : (flush ? k_dedisperse<uint8_t, true, false>
                                   : k_dedisperse<uint8_t, false, false>);
        PSX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        kern<<<grid, kDdThreads, smem, st>>>(a);
    }
    return launch_status("k_dedisperse");
}

}  // namespace

extern "C" {

int psx_dedisp_create(size_t nchans, float tsamp, float fch1, float foff, psx_dedisp_plan** out)
{
    clear_error();
    if (!out || nchans == 0 || nchans > (1u << 20) || !(tsamp > 0.0f) || !(fch1 > 0.0f) ||
        !(foff < 0.0f) || !(fch1 + (float)(nchans - 1) * foff > 0.0f)) {
        set_error("psx_dedisp_create: need nchans > 0, tsamp > 0 and a band fch1 > ... > 0 "
                  "with foff < 0");
        return PSX_ERR_INVALID;
    }
    auto* p = new (std::nothrow) psx_dedisp_plan();
    if (!p) return PSX_ERR_ALLOC;
    p->nchans = nchans;
    p->tsamp = tsamp;
    p->fch1 = fch1;
    p->foff = foff;
    p->delays.resize(nchans);
    for (size_t c = 0; c < nchans; ++c) {
        float inv_f = 1.0f / (fch1 + (float)c * foff);
        float inv_0 = 1.0f / fch1;
        float diff = inv_f * inv_f - inv_0 * inv_0;
        p->delays[c] = (float)((double)kDmConst / (double)tsamp * (double)diff);
    }
    p->live.assign(nchans, 1);
    *out = p;
    return PSX_OK;
}

int psx_dedisp_destroy(psx_dedisp_plan* plan)
{
    delete plan;
    return PSX_OK;
}

int psx_dedisp_set_dm_list(psx_dedisp_plan* p, const float* h_dms, size_t n)
{
    clear_error();
    if (!p || (!h_dms && n) || n == 0) {
        set_error("psx_dedisp_set_dm_list: empty list");
        return PSX_ERR_INVALID;
    }
    for (size_t i = 0; i < n; ++i)
        if (!(h_dms[i] >= 0.0f) || !std::isfinite(h_dms[i])) {
            set_error("psx_dedisp_set_dm_list: DM %zu is negative or not finite", i);
            return PSX_ERR_INVALID;
        }
    p->dms.assign(h_dms, h_dms + n);
    p->dirty = true;
    return PSX_OK;
}

int psx_dedisp_generate_dm_list(psx_dedisp_plan* p, float dm_start, float dm_end, float width_us,
                                float tol)
{
    clear_error();
    if (!p || !(dm_start >= 0.0f) || !(tol > 1.0f) || !(width_us >= 0.0f)) {
        set_error("psx_dedisp_generate_dm_list: need dm_start >= 0, tol > 1, width >= 0");
        return PSX_ERR_INVALID;
    }
    // next DM x from the previous p: t^2 + w^2 + a^2 x^2 + b^2 (x - p)^2
    // = tol^2 (t^2 + w^2 + a^2 p^2), times in microseconds; a is the
    // smearing across one channel per unit DM (8.3 us * foff / f_GHz^3) and
    // b = a * nchans / 4 that of a DM step across a quarter of the band
    const double ts = (double)p->tsamp * 1e6;
    const double f = ((double)p->fch1 + ((double)(p->nchans / 2) - 0.5) * (double)p->foff) * 1e-3;
    const double t2 = (double)tol * (double)tol;
    const double a = 8.3 * (double)p->foff / (f * f * f);
    const double a2 = a * a;
    const double b2 = a2 * ((double)(p->nchans * p->nchans) / 16.0);
    const double c = (ts * ts + (double)width_us * (double)width_us) * (t2 - 1.0);
    std::vector<float> list{dm_start};
    while (list.back() < dm_end) {
        double prev = (double)list.back();
        double k = c + t2 * a2 * prev * prev;
        double x = (b2 * prev + std::sqrt(-a2 * b2 * prev * prev + (a2 + b2) * k)) / (a2 + b2);
        list.push_back((float)x);
        if (list.size() > 100000000u || !(list.back() > list[list.size() - 2])) {
            set_error("psx_dedisp_generate_dm_list: the DM step does not advance");
            return PSX_ERR_INVALID;
        }
    }
    p->dms.swap(list);
    p->dirty = true;
    return PSX_OK;
}

size_t psx_dedisp_get_dm_count(const psx_dedisp_plan* p) { return p ? p->dms.size() : 0; }

int psx_dedisp_get_dm_list(const psx_dedisp_plan* p, float* h_out, size_t cap)
{
    clear_error();
    if (!p || !h_out) return PSX_ERR_INVALID;
    if (cap < p->dms.size()) {
        set_error("psx_dedisp_get_dm_list: %zu DMs do not fit in %zu", p->dms.size(), cap);
        return PSX_ERR_OVERFLOW;
    }
    std::copy(p->dms.begin(), p->dms.end(), h_out);
    return PSX_OK;
}

int psx_dedisp_get_delay_table(const psx_dedisp_plan* p, float* h_out)
{
    if (!p || !h_out) return PSX_ERR_INVALID;
    std::copy(p->delays.begin(), p->delays.end(), h_out);
    return PSX_OK;
}

int psx_dedisp_set_killmask(psx_dedisp_plan* p, const int* h_mask)
{
    if (!p) return PSX_ERR_INVALID;
    for (size_t c = 0; c < p->nchans; ++c) p->live[c] = h_mask ? (h_mask[c] != 0) : 1;
    p->dirty = true;
    return PSX_OK;
}

size_t psx_dedisp_get_max_delay(const psx_dedisp_plan* p) { return p ? p->max_delay() : 0; }

int psx_dedisp_set_scratch_limit(psx_dedisp_plan* p, size_t bytes)
{
    if (!p || bytes == 0) return PSX_ERR_INVALID;
    p->scratch_limit = bytes;
    return PSX_OK;
}

int psx_dedisp_execute(psx_dedisp_plan* p, size_t nsamps, const uint8_t* d_in, int nbits,
                       float* d_out, size_t out_pitch, int flags, psx_stream_t stream)
{
    clear_error();
    size_t nout = 0, pitch = 0, gulp = 0;
    PSX_TRY(check_input(p, nsamps, nbits, d_out, out_pitch, &nout));
    if (!d_in) return PSX_ERR_INVALID;
    cudaStream_t st = cs(stream);
    const int el = nbits == 16 ? 2 : 1;
    PSX_TRY(prepare(p, nout, el, st, &gulp, &pitch));
    const size_t row_bytes = p->nchans * (size_t)nbits / 8;
    const size_t md = p->max_delay();
    for (size_t g0 = 0; g0 < nout; g0 += gulp) {
        const size_t n = std::min(gulp, nout - g0);
        PSX_TRY(unpack(nbits, d_in + g0 * row_bytes, n + md, 0, pitch, p, pitch, st));
        PSX_TRY(dedisperse(p, nbits, pitch, n, d_out + g0, out_pitch, flags, st));
    }
    return PSX_OK;
}

int psx_dedisp_execute_host(psx_dedisp_plan* p, size_t nsamps, const uint8_t* h_in, int nbits,
                            float* d_out, size_t out_pitch, int flags, psx_stream_t stream)
{
    clear_error();
    size_t nout = 0, pitch = 0, gulp = 0;
    PSX_TRY(check_input(p, nsamps, nbits, d_out, out_pitch, &nout));
    if (!h_in) return PSX_ERR_INVALID;
    cudaStream_t st = cs(stream);
    const int el = nbits == 16 ? 2 : 1;
    PSX_TRY(prepare(p, nout, el, st, &gulp, &pitch));
    const size_t row_bytes = p->nchans * (size_t)nbits / 8;
    const size_t md = p->max_delay();
    // pieces of about 32 MB, a multiple of the unpack tile
    size_t rows = std::max<size_t>(kUpRows, (32u << 20) / row_bytes / kUpRows * kUpRows);
    rows = std::min(rows, round_up(std::min(gulp, nout) + md, kUpRows));
    PSX_TRY(grow(reinterpret_cast<void**>(&p->d_stage), &p->stage_cap, 2 * rows * row_bytes,
                 "input staging"));
    if (!p->copy_stream) {
        PSX_CUDA(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            PSX_CUDA(cudaEventCreateWithFlags(&p->ev_copied[i], cudaEventDisableTiming));
            PSX_CUDA(cudaEventCreateWithFlags(&p->ev_used[i], cudaEventDisableTiming));
        }
    }
    // the copy stream starts after what `stream` already holds (the
    // staging buffers may still be read by an earlier call)
    PSX_CUDA(cudaEventRecord(p->ev_used[0], st));
    PSX_CUDA(cudaEventRecord(p->ev_used[1], st));
    size_t k = 0;
    for (size_t g0 = 0; g0 < nout; g0 += gulp) {
        const size_t n_out = std::min(gulp, nout - g0);
        const size_t n_in = n_out + md;
        for (size_t r0 = 0; r0 < n_in; r0 += rows, ++k) {
            const int b = (int)(k & 1);
            const size_t n = std::min(rows, n_in - r0);
            uint8_t* buf = p->d_stage + (size_t)b * rows * row_bytes;
            PSX_CUDA(cudaStreamWaitEvent(p->copy_stream, p->ev_used[b], 0));
            PSX_CUDA(cudaMemcpyAsync(buf, h_in + (g0 + r0) * row_bytes, n * row_bytes,
                                     cudaMemcpyHostToDevice, p->copy_stream));
            PSX_CUDA(cudaEventRecord(p->ev_copied[b], p->copy_stream));
            PSX_CUDA(cudaStreamWaitEvent(st, p->ev_copied[b], 0));
            const bool last = r0 + n >= n_in;
            PSX_TRY(unpack(nbits, buf, n, r0, last ? pitch - r0 : n, p, pitch, st));
            PSX_CUDA(cudaEventRecord(p->ev_used[b], st));
        }
        PSX_TRY(dedisperse(p, nbits, pitch, n_out, d_out + g0, out_pitch, flags, st));
    }
    return PSX_OK;
}

}  // extern "C"
