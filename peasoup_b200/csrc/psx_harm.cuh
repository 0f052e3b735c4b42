// psx_harm.cuh -- fused fractional harmonic summing, threshold test and
// compaction for the search loop (reference src/kernels.cu:34-100 and the
// copy_if of src/kernels.cu:398-423, fused).
//
// One CTA handles a tile of T consecutive output bins [i0, i0+T) of one
// spectrum (i0 a multiple of 128).  The fraction m/2^h of output bin
// i0+j is input bin (i0*m >> h) + ((j*m + 2^(h-1)) >> h): every fraction
// reads one contiguous window of about T*m/2^h bins that starts at the
// exact integer i0*m/2^h.  The CTA stages the tile and the 2^F - 1
// windows in shared memory with 128-bit loads, then each thread sums its
// outputs with shared loads at per-fraction base offsets plus
// compile-time immediates, in the reference's summation order, tests each
// fold against the threshold inside its search range and appends the hits
// with one atomic per warp and fold.
#pragma once
#include <cuda_runtime.h>
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

template <int Q, int F, int T, int BD>
struct FracStep {
    // Adds fraction Q to every output of this thread (K outputs), emitting
    // at fold boundaries, then recurses to fraction Q+1.
    static __device__ __forceinline__ void run(const float* __restrict__ sm, float (&val)[T / BD],
                                               const unsigned (&base)[nfrac(F) > 0 ? nfrac(F) : 1],
                                               unsigned i0, unsigned tid, unsigned lane,
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
            for (int k = 0; k < T / BD; ++k) {
                const unsigned i = i0 + tid + k * BD;
                const float s = fold_scale<h>(val[k]);
                const bool hit = (int)i >= pp.start[h] && (int)i < pp.end[h] && s > pp.thresh;
                emit_hit(hit, trial, h, i, s, rec, counter, cap, lane);
            }
        }
        FracStep<Q + 1, F, T, BD>::run(sm, val, base, i0, tid, lane, pp, trial, rec, counter, cap);
    }
};

template <int F, int T, int BD>
struct FracStep<(1 << F) - 1, F, T, BD> {
    static __device__ __forceinline__ void run(const float*, float (&)[T / BD],
                                               const unsigned (&)[nfrac(F) > 0 ? nfrac(F) : 1],
                                               unsigned, unsigned, unsigned, const PeakParams&,
                                               int, int4*, unsigned*, unsigned)
    {
    }
};

template <int F, int T, int BD>
__global__ void __launch_bounds__(BD) k_harm_tiles(const float* __restrict__ p, size_t ppitch,
                                                   unsigned row_len, PeakParams pp, int trial0,
                                                   int4* __restrict__ rec,
                                                   unsigned* __restrict__ counter, unsigned cap)
{
    static_assert(T % 128 == 0 && BD % 32 == 0 && T % BD == 0, "tile shape");
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const int trial = trial0 + (int)blockIdx.y;
    const float* __restrict__ row = p + (size_t)blockIdx.y * ppitch;
    const float4* __restrict__ row4 = reinterpret_cast<const float4*>(row);
    const unsigned tid = threadIdx.x, lane = tid & 31u;
    const unsigned i0 = pp.lo + blockIdx.x * T;
    const unsigned len4 = row_len / 4;

    // ---- stage the tile and every fraction's window (128-bit loads)
    {
        const unsigned a4 = i0 / 4;
        for (unsigned j = tid; j < T / 4; j += BD) {
            const unsigned g = a4 + j;
            smem4[j] = g < len4 ? row4[g] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    // fully unrolled: every fraction's slot offset and shape is a
    // compile-time constant
#pragma unroll
    for (int q = 0; q < nfrac(F); ++q) {
        const unsigned h = (unsigned)frac_h(q), m = (unsigned)frac_m(q);
        const unsigned a = (unsigned)(((unsigned long long)i0 * m) >> h);
        const unsigned last = a + (unsigned)((((unsigned long long)(T - 1) * m) + (1u << (h - 1))) >> h);
        const unsigned a4 = a & ~3u;
        const unsigned n4 = (last + 1 - a4 + 3) / 4;
        float4* dst = smem4 + slot_offset(q, T) / 4;
        for (unsigned j = tid; j < n4; j += BD) {
            const unsigned g = a4 / 4 + j;
            dst[j] = g < len4 ? row4[g] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    __syncthreads();

    // ---- per-thread base offsets of each fraction
    constexpr int NF = nfrac(F) > 0 ? nfrac(F) : 1;
    unsigned base[NF];
#pragma unroll
    for (int q = 0; q < nfrac(F); ++q) {
        const unsigned h = (unsigned)frac_h(q), m = (unsigned)frac_m(q);
        const unsigned a = (unsigned)(((unsigned long long)i0 * m) >> h);
        base[q] = (unsigned)slot_offset(q, T) + (a & 3u) + ((tid * m + (1u << (h - 1))) >> h);
    }

    // ---- fold 0 and the running sums
    float val[T / BD];
#pragma unroll
    for (int k = 0; k < T / BD; ++k) {
        const unsigned j = tid + k * BD, i = i0 + j;
        val[k] = sm[j];
        const bool hit = (int)i >= pp.start[0] && (int)i < pp.end[0] && val[k] > pp.thresh;
        emit_hit(hit, trial, 0, i, val[k], rec, counter, cap, lane);
    }
    FracStep<0, F, T, BD>::run(sm, val, base, i0, tid, lane, pp, trial, rec, counter, cap);
}

}  // namespace psx
