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
template <int H>
__device__ __forceinline__ void test_and_emit(float s, const PeakParams& pp, unsigned i,
                                              int trial, int4* __restrict__ rec,
                                              unsigned* __restrict__ counter, unsigned cap,
                                              unsigned lane)
{
    const bool over = s > pp.thresh;
    if (__any_sync(0xffffffffu, over)) {
        const bool hit = over && (int)i >= pp.start[H] && (int)i < pp.end[H];
        emit_hit(hit, trial, H, i, s, rec, counter, cap, lane);
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
                test_and_emit<h>(fold_scale<h>(val[k]), pp, i0 + tid + k * BD, trial, rec,
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

// Per-fraction copy parameters, indexed by lane (lane 0 = the tile):
// numerator, log2 denominator and shared-memory offset of the slot.
template <int T>
struct WindowTable {
    int m[32], h[32], off[32];
    constexpr WindowTable() : m(), h(), off()
    {
        m[0] = 1;
        h[0] = 0;
        off[0] = 0;
        for (int q = 0; q < 31; ++q) {
            m[q + 1] = frac_m(q);
            h[q + 1] = frac_h(q);
            off[q + 1] = slot_offset(q, T);
        }
    }
};

// Stage item `i0` of `row` into the stage buffer `sm`: warp 0 issues one
// bulk copy per lane (lane 0 the tile, lane q+1 fraction q) after lane 0
// armed `bar` with the total byte count; parts past the row end are
// zero-filled by all threads.  The caller guarantees the buffer is free.
template <int F, int T, int BD>
__device__ __forceinline__ void stage_item(float* sm, uint64_t* bar, const float* __restrict__ row,
                                           unsigned row_len, unsigned i0, unsigned tid,
                                           const WindowTable<T>& W)
{
    constexpr int NW = nfrac(F) + 1;
    if (tid < 32) {
        const unsigned lane = tid;
        unsigned a4 = 0, len = 0;
        if (lane < (unsigned)NW) {
            const unsigned m = (unsigned)W.m[lane], h = (unsigned)W.h[lane];
            // i0 is a multiple of 128, so i0*m/2^h is a multiple of 4
            a4 = (unsigned)(((unsigned long long)i0 * m) >> h);
            const unsigned n = lane == 0 ? (unsigned)T
                                         : (unsigned)(((((unsigned long long)(T - 1) * m) +
                                                        (1u << (h - 1))) >> h) + 4u) & ~3u;
            len = a4 < row_len ? min(n, row_len - a4) : 0u;
        }
        const unsigned total = __reduce_add_sync(0xffffffffu, 4u * len);
        if (lane == 0) mbar_arrive_expect_tx(bar, total);
        __syncwarp();
        if (len) bulk_g2s(sm + W.off[lane], row + a4, 4u * len, bar);
    }
    if (i0 + T > row_len) {
        for (unsigned j = tid; j < (unsigned)T; j += BD)
            if (i0 + j >= row_len) sm[j] = 0.f;
#pragma unroll
        for (int q = 0; q < nfrac(F); ++q) {
            const unsigned a4 =
                (unsigned)(((unsigned long long)i0 * (unsigned)frac_m(q)) >> frac_h(q));
            for (unsigned j = tid; j < (unsigned)slot_floats(q, T); j += BD)
                if (a4 + j >= row_len) sm[slot_offset(q, T) + j] = 0.f;
        }
    }
}

template <int F, int T, int BD>
__device__ __forceinline__ void sum_item(const float* __restrict__ sm,
                                         const unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1],
                                         unsigned i0, unsigned tid, const PeakParams& pp,
                                         int trial, int4* __restrict__ rec,
                                         unsigned* __restrict__ counter, unsigned cap)
{
    float val[T / BD];
#pragma unroll
    for (int k = 0; k < T / BD; ++k) {
        val[k] = sm[tid + k * BD];
        test_and_emit<0>(val[k], pp, i0 + tid + k * BD, trial, rec, counter, cap, tid & 31u);
    }
    FracStep<0, F, T, BD>::run(sm, base, val, i0, tid, pp, trial, rec, counter, cap);
}

template <int T>
struct WindowTables {
    static __device__ const WindowTable<T>& get();
};

__constant__ WindowTable<512> kWindows512 = WindowTable<512>();
__constant__ WindowTable<1024> kWindows1024 = WindowTable<1024>();
template <> __device__ __forceinline__ const WindowTable<512>& WindowTables<512>::get() { return kWindows512; }
template <> __device__ __forceinline__ const WindowTable<1024>& WindowTables<1024>::get() { return kWindows1024; }

// Persistent CTA: work item w = (row, tile) taken round-robin; two stage
// buffers form a ring so the TMA engine stages item w+grid while the
// threads sum item w.  Items alternate between the stages, and the loop
// is unrolled by two so each stage's base is a compile-time offset.
template <int F, int T, int BD>
__global__ void __launch_bounds__(BD, 3) k_harm_tiles(const float* __restrict__ p, size_t ppitch,
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
    const WindowTable<T>& W = WindowTables<T>::get();
    const unsigned tid = threadIdx.x;
    const unsigned nitems = ntiles * (unsigned)rows;
    unsigned w = blockIdx.x;
    if (w >= nitems) return;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init_fence();
    }
    // item-independent part of every fraction's shared-memory offset
    unsigned base[nfrac(F) > 0 ? nfrac(F) : 1];
#pragma unroll
    for (int q = 0; q < nfrac(F); ++q) {
        const unsigned h = (unsigned)frac_h(q), m = (unsigned)frac_m(q);
        base[q] = (unsigned)slot_offset(q, T) + ((tid * m + (1u << (h - 1))) >> h);
    }
    __syncthreads();
    const unsigned lo = pp.lo;
#define PSX_ROW(it) (p + (size_t)((it) / ntiles) * ppitch)
#define PSX_I0(it) (lo + ((it) % ntiles) * (unsigned)T)
    stage_item<F, T, BD>(smem, &bar[0], PSX_ROW(w), row_len, PSX_I0(w), tid, W);
    unsigned ph0 = 0u, ph1 = 0u;
    bool ok = true;
    for (;;) {
        // ---- item in stage 0
        unsigned nxt = w + gridDim.x;
        if (nxt < nitems)
            stage_item<F, T, BD>(smem + STAGE, &bar[1], PSX_ROW(nxt), row_len, PSX_I0(nxt), tid, W);
        if (!mbar_wait_bounded(&bar[0], ph0, 1u << 22)) {
            ok = false;  // reported below; wait once more for the copies in flight
            mbar_wait_bounded(&bar[0], ph0, 1u << 22);
        }
        ph0 ^= 1u;
        sum_item<F, T, BD>(smem, base, PSX_I0(w), tid, pp, trial0 + (int)(w / ntiles), rec,
                           counter, cap);
        __syncthreads();  // stage 0 free
        w = nxt;
        if (w >= nitems) break;
        // ---- item in stage 1
        nxt = w + gridDim.x;
        if (nxt < nitems)
            stage_item<F, T, BD>(smem, &bar[0], PSX_ROW(nxt), row_len, PSX_I0(nxt), tid, W);
        if (!mbar_wait_bounded(&bar[1], ph1, 1u << 22)) {
            ok = false;  // reported below; wait once more for the copies in flight
            mbar_wait_bounded(&bar[1], ph1, 1u << 22);
        }
        ph1 ^= 1u;
        sum_item<F, T, BD>(smem + STAGE, base, PSX_I0(w), tid, pp, trial0 + (int)(w / ntiles),
                           rec, counter, cap);
        __syncthreads();  // stage 1 free
        w = nxt;
        if (w >= nitems) break;
    }
#undef PSX_ROW
#undef PSX_I0
    if (!ok && (tid & 31u) == 0) atomicExch(counter + 1, kHarmStagingTimeout);
}

}  // namespace psx
