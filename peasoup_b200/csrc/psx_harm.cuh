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

// Copy parameters of window `lane` (0 = the tile, q+1 = fraction q):
// numerator, log2 denominator and shared-memory offset, computed in
// registers (no table) from the fold structure: fold h has 2^(h-1)
// fractions; fold 2 lists 3/4 before 1/4, the other folds ascend.
template <int T>
__device__ __forceinline__ void window_params(unsigned lane, unsigned& m, unsigned& h,
                                              unsigned& off)
{
    if (lane == 0) {
        m = 1;
        h = 0;
        off = 0;
        return;
    }
    const unsigned q = lane - 1;                 // fraction index
    h = 32u - __clz(q + 1);                      // floor(log2(q+1)) + 1
    const unsigned first = (1u << (h - 1)) - 1;  // first fraction of fold h
    const unsigned r = q - first;                // position inside the fold
    m = (h == 2) ? (r == 0 ? 3u : 1u) : 2u * r + 1u;
    // slots of all earlier folds: sum over h' < h of (T*2^(h'-2) + 8*2^(h'-1))
    off = (unsigned)T;
    for (unsigned hh = 1; hh < h; ++hh) off += ((unsigned)T << hh >> 2) + (8u << (hh - 1));
    // earlier fractions of this fold: numerators sum to r^2 (3 for fold 2's second)
    const unsigned msum = (h == 2) ? (r == 0 ? 0u : 3u) : r * r;
    off += (((unsigned)T * msum) >> h) + 8u * r;
}

template <int F, int T, int NC>
__device__ __forceinline__ void sum_item(const float* __restrict__ sm,
                                         const unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1],
                                         unsigned i0, unsigned tid, const PeakParams& pp,
                                         int trial, int4* __restrict__ rec,
                                         unsigned* __restrict__ counter, unsigned cap)
{
    float val[T / NC];
#pragma unroll
    for (int k = 0; k < T / NC; ++k) {
        val[k] = sm[tid + k * NC];
        test_and_emit<0>(val[k], pp, i0 + tid + k * NC, trial, rec, counter, cap, tid & 31u);
    }
    FracStep<0, F, T, NC>::run(sm, base, val, i0, tid, pp, trial, rec, counter, cap);
}

// Persistent, warp-specialised CTA: warp 0 produces (bulk copies of item
// w into stage w%S once the consumers released it), warps 1..NC/32
// consume (sum, test, append), S stages in a ring.  Work items w = (row,
// tile) are taken round-robin over the grid.  full[s] completes when a
// stage's bytes have landed; empty[s] when every consumer warp has
// finished with it.  No CTA-wide barrier is used inside the loop; every
// wait is bounded and a timeout is reported in counter[1].
template <int F, int T, int NC, int S>
__global__ void __launch_bounds__(NC + 32, 3) k_harm_tiles(const float* __restrict__ p,
                                                           size_t ppitch, unsigned row_len,
                                                           PeakParams pp, int trial0, int rows,
                                                           unsigned ntiles,
                                                           int4* __restrict__ rec,
                                                           unsigned* __restrict__ counter,
                                                           unsigned cap)
{
    static_assert(T % 128 == 0 && NC % 32 == 0 && T % NC == 0, "tile shape");
    constexpr int STAGE = harm_smem_floats(F, T);
    constexpr int NW = nfrac(F) + 1;  // windows (tile + fractions)
    constexpr unsigned kLimit = 1u << 22;
    extern __shared__ float4 smem4[];
    __shared__ __align__(8) uint64_t full[S], empty[S];
    float* smem = reinterpret_cast<float*>(smem4);
    const unsigned nitems = ntiles * (unsigned)rows;
    if (blockIdx.x >= nitems) return;
    const unsigned warp = threadIdx.x / 32, lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NC / 32);
        }
        mbar_init_fence();
    }
    __syncthreads();
    bool ok = true;
    if (warp == 0) {
        // ---------------- producer
        unsigned m = 0, h = 0, off = 0;
        window_params<T>(lane, m, h, off);
        unsigned j = 0;
        for (unsigned w = blockIdx.x; w < nitems; w += gridDim.x, ++j) {
            const unsigned s = j % S;
            if (j >= (unsigned)S) {  // wait until the consumers released stage s
                const unsigned ph = ((j / S) - 1) & 1u;
                if (!mbar_wait_bounded(&empty[s], ph, kLimit)) ok = false;
            }
            float* sm = smem + s * STAGE;
            const float* row = p + (size_t)(w / ntiles) * ppitch;
            const unsigned i0 = pp.lo + (w % ntiles) * (unsigned)T;
            unsigned a4 = 0, len = 0;
            if (lane < (unsigned)NW) {
                // i0 is a multiple of 128, so i0*m/2^h is a multiple of 4
                a4 = (unsigned)(((unsigned long long)i0 * m) >> h);
                const unsigned n =
                    lane == 0 ? (unsigned)T
                              : ((unsigned)((((unsigned long long)(T - 1) * m) + (1u << (h - 1))) >> h) + 4u) & ~3u;
                len = a4 < row_len ? min(n, row_len - a4) : 0u;
                // past the row end (last tile only): zero-fill this window's slot
                if (a4 + (lane == 0 ? (unsigned)T : n) > row_len)
                    for (unsigned k = len; k < (lane == 0 ? (unsigned)T : n); ++k) sm[off + k] = 0.f;
            }
            const unsigned total = __reduce_add_sync(0xffffffffu, 4u * len);
            __syncwarp();
            if (lane == 0) mbar_arrive_expect_tx(&full[s], total);
            __syncwarp();
            if (len) bulk_g2s(sm + off, row + a4, 4u * len, &full[s]);
        }
        // the consumers wait for every stage they use; nothing is left in
        // flight once they are done, so the producer simply ends here
    } else {
        // ---------------- consumers
        const unsigned tid = threadIdx.x - 32;
        unsigned base[nfrac(F) > 0 ? nfrac(F) : 1];
#pragma unroll
        for (int q = 0; q < nfrac(F); ++q) {
            const unsigned hh = (unsigned)frac_h(q), mm = (unsigned)frac_m(q);
            base[q] = (unsigned)slot_offset(q, T) + ((tid * mm + (1u << (hh - 1))) >> hh);
        }
        unsigned j = 0;
        for (unsigned w = blockIdx.x; w < nitems; w += gridDim.x, ++j) {
            const unsigned s = j % S;
            const unsigned ph = (j / S) & 1u;
            if (!mbar_wait_bounded(&full[s], ph, kLimit)) {
                ok = false;
                mbar_wait_bounded(&full[s], ph, kLimit);  // let the copies land
            }
            const unsigned i0 = pp.lo + (w % ntiles) * (unsigned)T;
            sum_item<F, T, NC>(smem + s * STAGE, base, i0, tid, pp, trial0 + (int)(w / ntiles),
                               rec, counter, cap);
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[s])) : "memory");
        }
    }
    if (!ok && lane == 0) atomicExch(counter + 1, kHarmStagingTimeout);
}

}  // namespace psx
