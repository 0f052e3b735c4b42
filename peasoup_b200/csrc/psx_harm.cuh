// psx_harm.cuh -- fused fractional harmonic summing, threshold test and
// compaction for the search loop (reference src/kernels.cu:34-100 and the
// copy_if of src/kernels.cu:398-423, fused).
//
// Work item: a tile of T consecutive output bins [i0, i0+T) of one
// spectrum (i0 a multiple of 128).  The fraction m/2^h of output bin i0+j
// is input bin (i0*m >> h) + ((j*m + 2^(h-1)) >> h): every fraction reads
// one contiguous window of about T*m/2^h bins that starts at the exact
// integer i0*m/2^h.  One thread stages the tile and the 2^F - 1 windows
// into shared memory with bulk asynchronous copies (the TMA engine)
// completing on an mbarrier; every thread then sums its outputs with
// shared loads at per-fraction base offsets plus compile-time immediates,
// in the reference's summation order.  CTAs are persistent and keep two
// stages, so the copies of the next item overlap the sums of this one.
//
// Threshold crossings are rare: each fold's test is one warp vote, and the
// search-range check and the append (one atomic per warp and fold) run
// only in warps where some lane crossed.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "psx_device.cuh"

namespace psx {

struct PeakParams {
    int start[6];
    int end[6];
    unsigned lo, hi;  // union of the ranges; lo is rounded down to 128
    float thresh;
};

// Fraction q (0-based) in the reference's order: fold 1 {1/2}; fold 2
// {3/4, 1/4}; folds 3..5 {1/2^h, 3/2^h, ...} ascending.
__host__ __device__ constexpr int frac_h(int q)
{
    return q < 1 ? 1 : q < 3 ? 2 : q < 7 ? 3 : q < 15 ? 4 : 5;
}
__host__ __device__ constexpr int frac_m(int q)
{
    return q == 0 ? 1 : q == 1 ? 3 : q == 2 ? 1 : q < 7 ? 2 * (q - 3) + 1
                                            : q < 15 ? 2 * (q - 7) + 1 : 2 * (q - 15) + 1;
}
__host__ __device__ constexpr int nfrac(int F) { return (1 << F) - 1; }
// Last fraction of fold h.
__host__ __device__ constexpr int fold_last(int h) { return (1 << h) - 2; }
// Shared-memory slot (floats) of fraction q: the window plus alignment slack.
__host__ __device__ constexpr int slot_floats(int q, int T)
{
    return ((T * frac_m(q)) >> frac_h(q)) + 8;
}
__host__ __device__ constexpr int slot_offset(int q, int T)
{
    int off = T;
    for (int r = 0; r < q; ++r) off += slot_floats(r, T);
    return off;
}
__host__ __device__ constexpr int harm_smem_floats(int F, int T)
{
    return slot_offset(nfrac(F), T);
}

// ---- bulk asynchronous copy (TMA engine) and mbarrier helpers ---------
__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing as transaction bytes on `bar`.  Not
// multicast: the destination is this CTA's own shared memory.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Bounded wait: gives up after `limit` polls (each poll may suspend the
// thread for a hardware-defined time) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase, unsigned limit)
{
    for (unsigned it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// Status written to counter[1] when staging could not complete (the
// engine keeps its hit count in counter[0] and this error word next to it).
constexpr unsigned kHarmStagingTimeout = 0x5441u;

__device__ __forceinline__ void emit_hit(bool hit, int trial, int fold, unsigned bin, float val,
                                         int4* __restrict__ rec, unsigned* __restrict__ counter,
                                         unsigned cap, unsigned lane)
{
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (m == 0u) return;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if ((int)lane == leader) base = atomicAdd(counter, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (hit) {
        const unsigned pos = base + __popc(m & ((1u << lane) - 1u));
        if (pos < cap) rec[pos] = make_int4(trial, fold, (int)bin, __float_as_int(val));
    }
}

template <int F>
__device__ __forceinline__ float fold_scale(float val);
// The reference scales the running float sum by a double factor and
// stores the float-rounded product (src/kernels.cu:46, 53, 62, 75, 96).
template <> __device__ __forceinline__ float fold_scale<1>(float val) { return val * rsqrt(2.0); }
template <> __device__ __forceinline__ float fold_scale<2>(float val) { return val * 0.5; }
template <> __device__ __forceinline__ float fold_scale<3>(float val) { return val * rsqrt(8.0); }
template <> __device__ __forceinline__ float fold_scale<4>(float val) { return val * 0.25; }
template <> __device__ __forceinline__ float fold_scale<5>(float val) { return val * rsqrt(32.0); }

// One warp-level threshold test: the range check and the append only run
// in warps where some lane crossed the threshold (rare).
__device__ __forceinline__ void test_and_emit(float s, const PeakParams& pp, int h, unsigned i,
                                              int trial, int4* __restrict__ rec,
                                              unsigned* __restrict__ counter, unsigned cap,
                                              unsigned lane)
{
    const bool over = s > pp.thresh;
    if (__any_sync(0xffffffffu, over)) {
        const bool hit = over && (int)i >= pp.start[h] && (int)i < pp.end[h];
        emit_hit(hit, trial, h, i, s, rec, counter, cap, lane);
    }
}

// Adds fraction Q to every output of the thread (K = T/BD outputs, BD
// apart), tests and emits at fold boundaries, recurses to Q+1.
template <int Q, int F, int T, int BD>
struct FracStep {
    static __device__ __forceinline__ void run(const float* __restrict__ sm,
                                               const unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1],
                                               float (&val)[T / BD], unsigned i0, unsigned tid,
                                               const PeakParams& pp, int trial,
                                               int4* __restrict__ rec,
                                               unsigned* __restrict__ counter, unsigned cap)
    {
        constexpr int h = frac_h(Q), m = frac_m(Q);
        constexpr int step = (BD * m) >> h;  // exact: BD is a multiple of 32
#pragma unroll
        for (int k = 0; k < T / BD; ++k) val[k] += sm[base[Q] + k * step];
        if (Q == fold_last(h)) {
#pragma unroll
            for (int k = 0; k < T / BD; ++k)
                test_and_emit(fold_scale<h>(val[k]), pp, h, i0 + tid + k * BD, trial, rec,
                              counter, cap, tid & 31u);
        }
        FracStep<Q + 1, F, T, BD>::run(sm, base, val, i0, tid, pp, trial, rec, counter, cap);
    }
};

template <int F, int T, int BD>
struct FracStep<(1 << F) - 1, F, T, BD> {
    static __device__ __forceinline__ void run(const float*, const unsigned (&)[nfrac(F) > 0 ? nfrac(F) : 1],
                                               float (&)[T / BD], unsigned, unsigned,
                                               const PeakParams&, int, int4*, unsigned*, unsigned)
    {
    }
};

// Stage tile `i0` of `row` into the buffer `sm` (thread 0 issues the bulk
// copies onto `bar`; everything past the row end is zero-filled by all
// threads).  The caller guarantees the buffer is free.
template <int F, int T, int BD>
__device__ __forceinline__ void stage_tile(float* sm, uint64_t* bar, const float* __restrict__ row,
                                           unsigned row_len, unsigned i0, unsigned tid)
{
    if (tid == 0) {
        unsigned lens[nfrac(F) + 1];
        unsigned bytes = 0;
        lens[0] = i0 < row_len ? min((unsigned)T, row_len - i0) : 0u;
        bytes += 4u * lens[0];
#pragma unroll
        for (int q = 0; q < nfrac(F); ++q) {
            const unsigned h = (unsigned)frac_h(q), m = (unsigned)frac_m(q);
            const unsigned a = (unsigned)(((unsigned long long)i0 * m) >> h);
            const unsigned last = a + (unsigned)((((unsigned long long)(T - 1) * m) + (1u << (h - 1))) >> h);
            const unsigned a4 = a & ~3u;
            const unsigned n = ((last + 1 - a4) + 3u) & ~3u;
            lens[q + 1] = a4 < row_len ? min(n, row_len - a4) : 0u;
            bytes += 4u * lens[q + 1];
        }
        mbar_arrive_expect_tx(bar, bytes);
        if (lens[0]) bulk_g2s(sm, row + i0, 4u * lens[0], bar);
#pragma unroll
        for (int q = 0; q < nfrac(F); ++q) {
            const unsigned h = (unsigned)frac_h(q), m = (unsigned)frac_m(q);
            const unsigned a4 = (unsigned)(((unsigned long long)i0 * m) >> h) & ~3u;
            if (lens[q + 1]) bulk_g2s(sm + slot_offset(q, T), row + a4, 4u * lens[q + 1], bar);
        }
    }
    if (i0 + T > row_len) {
        for (unsigned j = tid; j < (unsigned)T; j += BD)
            if (i0 + j >= row_len) sm[j] = 0.f;
#pragma unroll
        for (int q = 0; q < nfrac(F); ++q) {
            const unsigned h = (unsigned)frac_h(q), m = (unsigned)frac_m(q);
            const unsigned a4 = (unsigned)(((unsigned long long)i0 * m) >> h) & ~3u;
            for (unsigned j = tid; j < (unsigned)slot_floats(q, T); j += BD)
                if (a4 + j >= row_len) sm[slot_offset(q, T) + j] = 0.f;
        }
    }
}

// Persistent CTA: work item w = (row, tile) taken round-robin; two shared
// buffers form a ring so the TMA engine stages item w+1 while the threads
// sum item w.
template <int F, int T, int BD>
__global__ void __launch_bounds__(BD) k_harm_tiles(const float* __restrict__ p, size_t ppitch,
                                                   unsigned row_len, PeakParams pp, int trial0,
                                                   int rows, unsigned ntiles,
                                                   int4* __restrict__ rec,
                                                   unsigned* __restrict__ counter, unsigned cap)
{
    static_assert(T % 128 == 0 && BD % 32 == 0 && T % BD == 0, "tile shape");
    constexpr int STAGE = harm_smem_floats(F, T);
    extern __shared__ float4 smem4[];
    __shared__ __align__(8) uint64_t bar[2];
    float* smem = reinterpret_cast<float*>(smem4);
    const unsigned tid = threadIdx.x;
    const unsigned nitems = ntiles * (unsigned)rows;
    unsigned w = blockIdx.x;
    if (w >= nitems) return;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    auto item_row = [&](unsigned it) { return it / ntiles; };
    auto item_i0 = [&](unsigned it) { return pp.lo + (it % ntiles) * (unsigned)T; };
    stage_tile<F, T, BD>(smem, &bar[0], p + (size_t)item_row(w) * ppitch, row_len, item_i0(w), tid);
    unsigned phases = 0u;  // bit b: parity of the next completion of bar[b]
    for (unsigned j = 0; w < nitems; ++j, w += gridDim.x) {
        const unsigned cur = j & 1u;
        const unsigned nxt = w + gridDim.x;
        if (nxt < nitems)  // the other buffer was released at the end of the last item
            stage_tile<F, T, BD>(smem + (cur ^ 1u) * STAGE, &bar[cur ^ 1u],
                                 p + (size_t)item_row(nxt) * ppitch, row_len, item_i0(nxt), tid);
        const unsigned ph = (phases >> cur) & 1u;
        const bool staged = mbar_wait_bounded(&bar[cur], ph, 1u << 22);
        phases ^= 1u << cur;
        if (!__syncthreads_and(staged)) {
            // copies still in flight get a second bounded wait, then leave
            if (!staged) mbar_wait_bounded(&bar[cur], ph, 1u << 22);
            if (nxt < nitems) mbar_wait_bounded(&bar[cur ^ 1u], (phases >> (cur ^ 1u)) & 1u, 1u << 22);
            if (tid == 0) atomicExch(counter + 1, kHarmStagingTimeout);
            return;
        }
        const float* sm = smem + cur * STAGE;
        const unsigned i0 = item_i0(w);
        const int trial = trial0 + (int)item_row(w);
        unsigned base[nfrac(F) > 0 ? nfrac(F) : 1];
#pragma unroll
        for (int q = 0; q < nfrac(F); ++q) {
            const unsigned h = (unsigned)frac_h(q), m = (unsigned)frac_m(q);
            const unsigned a = (unsigned)(((unsigned long long)i0 * m) >> h);
            base[q] = (unsigned)slot_offset(q, T) + (a & 3u) + ((tid * m + (1u << (h - 1))) >> h);
        }
        float val[T / BD];
#pragma unroll
        for (int k = 0; k < T / BD; ++k) {
            val[k] = sm[tid + k * BD];
            test_and_emit(val[k], pp, 0, i0 + tid + k * BD, trial, rec, counter, cap, tid & 31u);
        }
        FracStep<0, F, T, BD>::run(sm, base, val, i0, tid, pp, trial, rec, counter, cap);
        __syncthreads();  // buffer `cur` is free for item j+2
    }
}

}  // namespace psx
