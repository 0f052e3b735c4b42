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
// Each consumer thread owns K = T/NC outputs (NC apart), accumulated in
// pairs with packed two-lane float adds (add.rn.f32x2: each lane rounds as
// a scalar add, so the sums are those of the reference's order).
// Threshold crossings are rare: a fast pass keeps each output's largest
// fold value, scaled in float, and votes against a threshold lowered by
// 2^-20 relative (the float scale is within 3*2^-24 of the reference's
// double-scaled product); only warps where some lane passes the vote run
// the exact pass (reference scales, search ranges, one atomic per warp and
// fold).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "psx_device.cuh"

namespace psx {

struct PeakParams {
    int start[6];
    int end[6];
    unsigned lo, hi;  // union of the ranges; lo is rounded down to 128
    float thresh;
    float vote;       // fast-pass vote level: thresh lowered by 2^-20 relative
    unsigned wait_limit;  // polls of one bounded barrier wait (kHarmWaitLimit)
    unsigned flags;       // kHarmNoCopies: stage nothing (every wait runs out)
};

// Default bound of one barrier wait (polls; each may suspend briefly).
constexpr unsigned kHarmWaitLimit = 1u << 22;
// Test hook: the producer arrives on the stage barriers but issues no
// copies, so the consumers' waits run out and the timeout path runs
// (no fault: every wait is bounded and nothing is left in flight).
constexpr unsigned kHarmNoCopies = 1u;

// Packed two-lane float arithmetic (sm_100): one instruction for two
// independent IEEE round-to-nearest operations.
__device__ __forceinline__ float2 f2add(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rc, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rc;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 f2mul(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rc, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rc;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}

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
// 16-byte aligned), completing as transaction bytes on `bar`.  The
// destination is this CTA's own shared memory only.
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

// Fold scales: the reference multiplies the running float sum by a double
// factor and stores the float-rounded product (src/kernels.cu:46, 53, 62,
// 75, 96).  For the factors 1/2 and 1/4 the double product is exact, so
// the float product x*0.5f / x*0.25f is the same correctly rounded value;
// the other three use the double factors rsqrt(2.0), rsqrt(8.0) and
// rsqrt(32.0), evaluated once per thread by the same function calls.
struct FoldScales {
    double r2, r8, r32;
    float f2, f8, f32;  // the same factors rounded to float (fast pass only)
    __device__ __forceinline__ FoldScales()
        : r2(rsqrt(2.0)), r8(rsqrt(8.0)), r32(rsqrt(32.0)),
          f2((float)r2), f8((float)r8), f32((float)r32) {}
};

// Float scale of fold H for the fast pass's vote.
template <int H>
__device__ __forceinline__ float fold_scale_f(const FoldScales& c)
{
    return H == 1 ? c.f2 : H == 2 ? 0.5f : H == 3 ? c.f8 : H == 4 ? 0.25f : c.f32;
}

template <int H>
__device__ __forceinline__ float fold_scale(float val, const FoldScales& c);
template <> __device__ __forceinline__ float fold_scale<1>(float val, const FoldScales& c) { return val * c.r2; }
template <> __device__ __forceinline__ float fold_scale<2>(float val, const FoldScales&) { return val * 0.5f; }
template <> __device__ __forceinline__ float fold_scale<3>(float val, const FoldScales& c) { return val * c.r8; }
template <> __device__ __forceinline__ float fold_scale<4>(float val, const FoldScales&) { return val * 0.25f; }
template <> __device__ __forceinline__ float fold_scale<5>(float val, const FoldScales& c) { return val * c.r32; }

// Adds fraction Q to every output of the thread (K = T/NC outputs, NC
// apart, accumulated as K/2 packed pairs).  At a fold boundary: in the fast
// pass (EMIT false) the float-scaled fold value only raises the running
// maximum `mx`; in the exact pass (EMIT true) the reference's scale and the
// fold's search range are applied and hits are appended with one atomic
// per warp.  Recurses to Q+1.
template <int Q, int F, int T, int NC, bool EMIT>
struct FracStep {
    static constexpr int K = T / NC;
    static __device__ __forceinline__ void run(const float* __restrict__ sm,
                                               const unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1],
                                               float2 (&acc)[K / 2], float (&mx)[K],
                                               const FoldScales& fs, unsigned i0, unsigned tid,
                                               const PeakParams& pp, int trial,
                                               int4* __restrict__ rec,
                                               unsigned* __restrict__ counter, unsigned cap)
    {
        constexpr int h = frac_h(Q), m = frac_m(Q);
        constexpr int step = (NC * m) >> h;  // exact: NC is a multiple of 32
#pragma unroll
        for (int k = 0; k < K / 2; ++k)
            acc[k] = f2add(acc[k], make_float2(sm[base[Q] + (2 * k) * step],
                                               sm[base[Q] + (2 * k + 1) * step]));
        if (Q == fold_last(h)) {
            if (EMIT) {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float v = (k & 1) ? acc[k / 2].y : acc[k / 2].x;
                    const float s = fold_scale<h>(v, fs);
                    const unsigned i = i0 + tid + k * NC;
                    const bool hit = s > pp.thresh && (int)i >= pp.start[h] && (int)i < pp.end[h];
                    emit_hit(hit, trial, h, i, s, rec, counter, cap, tid & 31u);
                }
            } else {
                const float sf = fold_scale_f<h>(fs);
#pragma unroll
                for (int k = 0; k < K / 2; ++k) {
                    const float2 s = f2mul(acc[k], make_float2(sf, sf));
                    mx[2 * k] = fmaxf(mx[2 * k], s.x);
                    mx[2 * k + 1] = fmaxf(mx[2 * k + 1], s.y);
                }
            }
        }
        FracStep<Q + 1, F, T, NC, EMIT>::run(sm, base, acc, mx, fs, i0, tid, pp, trial, rec,
                                             counter, cap);
    }
};

template <int F, int T, int NC, bool EMIT>
struct FracStep<(1 << F) - 1, F, T, NC, EMIT> {
    static __device__ __forceinline__ void run(const float*, const unsigned (&)[nfrac(F) > 0 ? nfrac(F) : 1],
                                               float2 (&)[T / NC / 2], float (&)[T / NC],
                                               const FoldScales&, unsigned, unsigned,
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

// The exact pass of one item (rare: only warps where some output passes
// the vote): every fold's value again with the reference's scales, its
// search range, and the appends.
template <int F, int T, int NC>
__device__ __forceinline__ void exact_body(const float* __restrict__ sm,
                                           const unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1],
                                           const FoldScales& fs, unsigned i0, unsigned tid,
                                           const PeakParams& pp, int trial, int4* __restrict__ rec,
                                           unsigned* __restrict__ counter, unsigned cap)
{
    constexpr int K = T / NC;
    float2 acc[K / 2];
    float mx[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const float v = sm[tid + k * NC];
        if (k & 1) acc[k / 2].y = v; else acc[k / 2].x = v;
        const unsigned i = i0 + tid + k * NC;
        const bool hit = v > pp.thresh && (int)i >= pp.start[0] && (int)i < pp.end[0];
        emit_hit(hit, trial, 0, i, v, rec, counter, cap, tid & 31u);
    }
    FracStep<0, F, T, NC, true>::run(sm, base, acc, mx, fs, i0, tid, pp, trial, rec, counter, cap);
}

// Shared-memory offset of fraction q's source for consumer `tid`.
template <int F, int T>
__device__ __forceinline__ void make_bases(unsigned tid,
                                           unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1])
{
#pragma unroll
    for (int q = 0; q < nfrac(F); ++q) {
        const unsigned hh = (unsigned)frac_h(q), mm = (unsigned)frac_m(q);
        base[q] = (unsigned)slot_offset(q, T) + ((tid * mm + (1u << (hh - 1))) >> hh);
    }
}

// The same, kept out of line so that the fast pass does not share its
// registers.  It rebuilds the offsets and scales itself: handing the fast
// pass's arrays to a call would give them an address and move them from
// registers to local memory for the fast pass too.
template <int F, int T, int NC>
__device__ __noinline__ void exact_pass_ool(const float* __restrict__ sm, unsigned i0,
                                            unsigned tid, const PeakParams& pp, int trial,
                                            int4* __restrict__ rec, unsigned* __restrict__ counter,
                                            unsigned cap)
{
    unsigned base[nfrac(F) > 0 ? nfrac(F) : 1];
    make_bases<F, T>(tid, base);
    const FoldScales fs;
    exact_body<F, T, NC>(sm, base, fs, i0, tid, pp, trial, rec, counter, cap);
}

// Sums one staged item: the fast pass, then -- only in warps where some
// output passes the vote -- the exact pass (inline or out of line).
template <int F, int T, int NC, int ROWS>
__device__ __noinline__ void exact_pass_rows_ool(const float* __restrict__ sm, unsigned i0,
                                                 unsigned tid, unsigned rho, const PeakParams& pp,
                                                 int trial, int4* __restrict__ rec,
                                                 unsigned* __restrict__ counter, unsigned cap);

template <int F, int T, int NC, bool OOL, int ROWS = 0>
__device__ __forceinline__ void sum_item(const float* __restrict__ sm,
                                         const unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1],
                                         const FoldScales& fs, unsigned i0, unsigned tid,
                                         const PeakParams& pp, int trial, int4* __restrict__ rec,
                                         unsigned* __restrict__ counter, unsigned cap,
                                         unsigned rho = 0)
{
    constexpr int K = T / NC;
    float2 acc[K / 2];
    float mx[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const float v = sm[tid + k * NC];
        if (k & 1) acc[k / 2].y = v; else acc[k / 2].x = v;
        mx[k] = v;
    }
    FracStep<0, F, T, NC, false>::run(sm, base, acc, mx, fs, i0, tid, pp, trial, rec, counter, cap);
    bool over = false;
#pragma unroll
    for (int k = 0; k < K; ++k) over |= mx[k] > pp.vote;
    if (__any_sync(0xffffffffu, over)) {
        if constexpr (ROWS > 0)
            exact_pass_rows_ool<F, T, NC, ROWS>(sm, i0, tid, rho, pp, trial, rec, counter, cap);
        else if (OOL)
            exact_pass_ool<F, T, NC>(sm, i0, tid, pp, trial, rec, counter, cap);
        else
            exact_body<F, T, NC>(sm, base, fs, i0, tid, pp, trial, rec, counter, cap);
    }
}

// Persistent, warp-specialised CTA: warp 0 produces (bulk copies of item
// w into stage w%2 once the consumers released it), the other NC/32 warps
// consume (sum, test, append); two stages form a ring.  Work items
// (row, tile) are taken round-robin over the grid.  full[s] completes when
// a stage's bytes have landed, empty[s] when every consumer warp is done
// with it.  No CTA-wide barrier is used in the loop; every wait is bounded
// (pp.wait_limit polls).  A wait that runs out sets a CTA-wide abort flag:
// both sides stop at their next item, the copies already issued are waited
// for (bounded) before the CTA exits, and counter[1] reports the timeout.
template <int F, int T, int NC, int MINB, bool OOL>
__global__ void __launch_bounds__(NC + 32, MINB) k_harm_tiles(const float* __restrict__ p,
                                                           size_t ppitch, unsigned row_len,
                                                           PeakParams pp, int trial0, int rows,
                                                           unsigned ntiles,
                                                           int4* __restrict__ rec,
                                                           unsigned* __restrict__ counter,
                                                           unsigned cap)
{
    static_assert(T % 128 == 0 && NC % 32 == 0 && T % (2 * NC) == 0, "tile shape");
    constexpr int STAGE = harm_smem_floats(F, T);
    constexpr int NW = nfrac(F) + 1;  // windows (tile + fractions)
    const unsigned kLimit = pp.wait_limit ? pp.wait_limit : kHarmWaitLimit;
    extern __shared__ float4 smem4[];
    __shared__ __align__(8) uint64_t full[2], empty[2];
    // abort: set by whoever's wait ran out, ends both loops at their next item;
    // issued/landed per stage let the CTA wait for its copies before exiting
    __shared__ volatile int abort_flag;
    __shared__ unsigned issued[2], landed[2];
    float* smem = reinterpret_cast<float*>(smem4);
    const unsigned nitems = ntiles * (unsigned)rows;
    if (blockIdx.x >= nitems) return;
    const unsigned warp = threadIdx.x / 32, lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NC / 32);
            issued[s] = 0;
            landed[s] = 0;
        }
        abort_flag = 0;
        mbar_init_fence();
    }
    __syncthreads();
    bool ok = true;
    // the item sequence of this CTA as (row, tile), advanced without division
    unsigned row = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
    const unsigned gstep_row = gridDim.x / ntiles, gstep_tile = gridDim.x % ntiles;
    auto advance = [&]() {
        row += gstep_row;
        tile += gstep_tile;
        if (tile >= ntiles) {
            tile -= ntiles;
            ++row;
        }
    };
    if (warp == 0) {
        // ---------------- producer
        unsigned m = 0, h = 0, off = 0;
        window_params<T>(lane, m, h, off);
        for (unsigned j = 0; row < (unsigned)rows; ++j, advance()) {
            const unsigned s = j & 1u;
            if (__any_sync(0xffffffffu, abort_flag != 0)) break;  // warp-uniform
            if (j >= 2) {  // wait until the consumers released stage s
                const bool got = mbar_wait_bounded(&empty[s], ((j >> 1) - 1) & 1u, kLimit);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    if (lane == 0) abort_flag = 1;
                    break;
                }
            }
            float* sm = smem + s * STAGE;
            const float* src = p + (size_t)row * ppitch;
            const unsigned i0 = pp.lo + tile * (unsigned)T;
            unsigned a4 = 0, len = 0;
            if (lane < (unsigned)NW) {
                // i0 is a multiple of 128, so i0*m/2^h is a multiple of 4
                a4 = (unsigned)(((unsigned long long)i0 * m) >> h);
                const unsigned n =
                    lane == 0 ? (unsigned)T
                              : ((unsigned)((((unsigned long long)(T - 1) * m) + (1u << (h - 1))) >> h) + 4u) & ~3u;
                len = a4 < row_len ? min(n, row_len - a4) : 0u;
                // past the row end (last tile only): zero-fill the rest of the slot
                for (unsigned k = len; k < n; ++k) sm[off + k] = 0.f;
            }
            const unsigned total = __reduce_add_sync(0xffffffffu, 4u * len);
            __syncwarp();
            if (lane == 0) mbar_arrive_expect_tx(&full[s], total);
            __syncwarp();
            if (pp.flags & kHarmNoCopies) continue;  // nothing staged, nothing in flight
            if (len) bulk_g2s(sm + off, src + a4, 4u * len, &full[s]);
            if (lane == 0) issued[s] += 1;
        }
    } else {
        // ---------------- consumers
        const unsigned tid = threadIdx.x - 32;
        const FoldScales fs;
        unsigned base[nfrac(F) > 0 ? nfrac(F) : 1];
        make_bases<F, T>(tid, base);
        unsigned ph = 0;
        for (;;) {
#pragma unroll
            for (unsigned s = 0; s < 2; ++s) {  // s is a compile-time stage index
                if (row >= (unsigned)rows || __any_sync(0xffffffffu, abort_flag != 0)) break;
                const bool got = mbar_wait_bounded(&full[s], ph, kLimit);
                if (!__all_sync(0xffffffffu, got)) {  // the warp decides together
                    ok = false;
                    if (lane == 0) abort_flag = 1;
                    break;
                }
                if (tid == 0) landed[s] += 1;
                sum_item<F, T, NC, OOL>(smem + s * STAGE, base, fs, pp.lo + tile * (unsigned)T,
                                        tid, pp, trial0 + (int)row, rec, counter, cap);
                __syncwarp();
                if (lane == 0)
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[s]))
                                 : "memory");
                advance();
            }
            if (row >= (unsigned)rows || __any_sync(0xffffffffu, abort_flag != 0)) break;
            ph ^= 1u;
        }
    }
    // After an abort, copies the producer issued may still be landing in this
    // CTA's shared memory: wait for them (bounded) before the CTA exits.
    __syncthreads();
    if (abort_flag && threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s)
            while (landed[s] < issued[s]) {
                if (!mbar_wait_bounded(&full[s], landed[s] & 1u, kLimit)) break;
                landed[s] += 1;
            }
    }
    if ((!ok || abort_flag) && lane == 0) atomicExch(counter + 1, kHarmStagingTimeout);
}

// ---------------------------------------------------------------------------
// Multi-row staging: one work item is one tile of T output bins for ROWS
// consecutive trials (rows of the spectrum buffer), and every window --
// the tile and each fraction's -- arrives for all ROWS rows at once as one
// 2D tensor copy (TMA) of a box [width, ROWS], so a CTA issues 2^F copies
// per ROWS * T outputs instead of per T.  The tensor maps view the buffer
// as rows of 8-byte elements (two floats), which keeps every window within
// the 256-element box limit (widths 32 .. 512 floats in steps of 32, one
// map each); window starts i0*m/2^h are multiples of 4 floats, i.e. 16
// bytes.  Bins past the row's end and rows past the buffer arrive as zeros
// (the maps' out-of-bounds fill), rows past the launch group's trials are
// staged but not summed.
constexpr int kHarmWidthClasses = 16;  // window widths 32 * (c + 1) floats

struct HarmMaps {
    CUtensorMap m[kHarmWidthClasses];
};

// Samples window q needs (q = -1: the tile) and its staged width.
__host__ __device__ constexpr int win_need(int q, int T)
{
    return q < 0 ? T : (((T - 1) * frac_m(q) + (1 << (frac_h(q) - 1))) >> frac_h(q)) + 1;
}
__host__ __device__ constexpr int win_width(int q, int T) { return (win_need(q, T) + 31) / 32 * 32; }
// Offset (floats) of window q's [ROWS][width] block in a stage; the tile's
// [ROWS][T] block comes first.
__host__ __device__ constexpr int rows_slot(int q, int T, int ROWS)
{
    int off = ROWS * T;
    for (int r = 0; r < q; ++r) off += ROWS * win_width(r, T);
    return q < 0 ? 0 : off;
}
__host__ __device__ constexpr int rows_stage_floats(int F, int T, int ROWS)
{
    return rows_slot(nfrac(F), T, ROWS);
}

// Offsets of fraction q's source for consumer `tid` of row `rho`, relative
// to that row's tile (sm + rho * T).
template <int F, int T, int ROWS>
__device__ __forceinline__ void make_bases_rows(unsigned tid, unsigned rho,
                                                unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1])
{
#pragma unroll
    for (int q = 0; q < nfrac(F); ++q) {
        const unsigned hh = (unsigned)frac_h(q), mm = (unsigned)frac_m(q);
        base[q] = (unsigned)rows_slot(q, T, ROWS) - rho * (unsigned)T +
                  rho * (unsigned)win_width(q, T) + ((tid * mm + (1u << (hh - 1))) >> hh);
    }
}

template <int F, int T, int NC, int ROWS>
__device__ __noinline__ void exact_pass_rows_ool(const float* __restrict__ sm, unsigned i0,
                                                 unsigned tid, unsigned rho, const PeakParams& pp,
                                                 int trial, int4* __restrict__ rec,
                                                 unsigned* __restrict__ counter, unsigned cap)
{
    unsigned base[nfrac(F) > 0 ? nfrac(F) : 1];
    make_bases_rows<F, T, ROWS>(tid, rho, base);
    const FoldScales fs;
    exact_body<F, T, NC>(sm, base, fs, i0, tid, pp, trial, rec, counter, cap);
}

// 2D tensor copy of the box at element coordinates (x, y) of `map` into
// this CTA's own shared memory only, completing as transaction bytes on
// `bar`.
__device__ __forceinline__ void tensor_g2s_2d(void* dst, const CUtensorMap* map, int x, int y,
                                              uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y),
          "r"(smem_addr(bar))
        : "memory");
}

// Persistent CTA (one per SM): warp 0 produces, ROWS * NC / 32 warps
// consume (NC per row); two stages.  Same ring, bounded waits and abort
// path as k_harm_tiles.
template <int F, int T, int NC, int ROWS>
__global__ void __launch_bounds__(ROWS * NC + 32, 1)
    k_harm_rows(const __grid_constant__ HarmMaps maps, PeakParams pp, int trial0, int rows,
                unsigned ntiles, int4* __restrict__ rec, unsigned* __restrict__ counter,
                unsigned cap)
{
    static_assert(T % 128 == 0 && NC % 32 == 0 && T % (2 * NC) == 0 && T <= 512, "tile shape");
    constexpr int STAGE = rows_stage_floats(F, T, ROWS);
    constexpr int NW = nfrac(F) + 1;          // windows (tile + fractions)
    constexpr unsigned NCW = ROWS * NC / 32;  // consumer warps
    const unsigned kLimit = pp.wait_limit ? pp.wait_limit : kHarmWaitLimit;
    extern __shared__ __align__(128) float4 smem4r[];
    __shared__ __align__(8) uint64_t full[2], empty[2];
    __shared__ volatile int abort_flag;
    __shared__ unsigned issued[2], landed[2];
    float* smem = reinterpret_cast<float*>(smem4r);
    const unsigned ngroups = ((unsigned)rows + ROWS - 1) / ROWS;
    const unsigned nitems = ntiles * ngroups;
    if (blockIdx.x >= nitems) return;
    const unsigned warp = threadIdx.x / 32, lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCW);
            issued[s] = 0;
            landed[s] = 0;
        }
        abort_flag = 0;
        mbar_init_fence();
    }
    __syncthreads();
    bool ok = true;
    unsigned grp = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
    const unsigned gstep_grp = gridDim.x / ntiles, gstep_tile = gridDim.x % ntiles;
    auto advance = [&]() {
        grp += gstep_grp;
        tile += gstep_tile;
        if (tile >= ntiles) {
            tile -= ntiles;
            ++grp;
        }
    };
    if (warp == 0) {
        // ---------------- producer: lane = window (0 the tile, q + 1 fraction q)
        const bool active = lane < (unsigned)NW;
        const int q = (int)lane - 1;
        unsigned m = 1, h = 0, slot = 0, wcls = 0, bytes = 0;
        if (active) {
            if (q >= 0) {
                m = (unsigned)frac_m(q);
                h = (unsigned)frac_h(q);
            }
            slot = (unsigned)rows_slot(q, T, ROWS);
            wcls = (unsigned)win_width(q, T) / 32u - 1u;
            bytes = 4u * (unsigned)ROWS * (unsigned)win_width(q, T);
        }
        const unsigned total = __reduce_add_sync(0xffffffffu, bytes);
        const CUtensorMap* map = &maps.m[wcls];
        for (unsigned j = 0; grp < ngroups; ++j, advance()) {
            const unsigned s = j & 1u;
            if (__any_sync(0xffffffffu, abort_flag != 0)) break;
            if (j >= 2) {
                const bool got = mbar_wait_bounded(&empty[s], ((j >> 1) - 1) & 1u, kLimit);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    if (lane == 0) abort_flag = 1;
                    break;
                }
            }
            if (lane == 0) mbar_arrive_expect_tx(&full[s], total);
            __syncwarp();
            if (pp.flags & kHarmNoCopies) continue;
            const unsigned i0 = pp.lo + tile * (unsigned)T;
            // window start in floats, a multiple of 4 (i0 is a multiple of 128)
            const unsigned a = (unsigned)(((unsigned long long)i0 * m) >> h);
            if (active)
                tensor_g2s_2d(smem + s * STAGE + slot, map, (int)(a >> 1), (int)(grp * ROWS),
                              &full[s]);
            if (lane == 0) issued[s] += 1;
        }
    } else {
        // ---------------- consumers: ROWS groups of NC threads, one row each
        const unsigned ct = threadIdx.x - 32;
        const unsigned rho = ct / NC, tid = ct % NC;  // rho is warp-uniform
        const FoldScales fs;
        unsigned base[nfrac(F) > 0 ? nfrac(F) : 1];
        make_bases_rows<F, T, ROWS>(tid, rho, base);
        unsigned ph = 0;
        for (;;) {
#pragma unroll
            for (unsigned s = 0; s < 2; ++s) {
                if (grp >= ngroups || __any_sync(0xffffffffu, abort_flag != 0)) break;
                const bool got = mbar_wait_bounded(&full[s], ph, kLimit);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    if (lane == 0) abort_flag = 1;
                    break;
                }
                if (ct == 0) landed[s] += 1;
                const unsigned row = grp * ROWS + rho;
                if (row < (unsigned)rows)
                    sum_item<F, T, NC, true, ROWS>(smem + s * STAGE + rho * T, base, fs,
                                                   pp.lo + tile * (unsigned)T, tid, pp,
                                                   trial0 + (int)row, rec, counter, cap, rho);
                __syncwarp();
                if (lane == 0)
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&empty[s]))
                                 : "memory");
                advance();
            }
            if (grp >= ngroups || __any_sync(0xffffffffu, abort_flag != 0)) break;
            ph ^= 1u;
        }
    }
    __syncthreads();
    if (abort_flag && threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s)
            while (landed[s] < issued[s]) {
                if (!mbar_wait_bounded(&full[s], landed[s] & 1u, kLimit)) break;
                landed[s] += 1;
            }
    }
    if ((!ok || abort_flag) && lane == 0) atomicExch(counter + 1, kHarmStagingTimeout);
}

}  // namespace psx
