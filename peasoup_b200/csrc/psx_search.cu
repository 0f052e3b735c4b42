// psx_search.cu -- the per-DM acceleration search engine behind
// psx_search_dm: the body of the reference's DM loop
// (src/pipeline_multi.cu:161-294) re-organised for a B200.
//
// Per DM (prologue, once):
//   H2D copy -> baseline removal -> zero padding -> R2C -> amplitude ->
//   5/25/125-bin running median fused with the division of the spectrum
//   -> birdie zapping -> interbin statistics (device-resident mean*N,
//   std*N) -> C2R into the resident dereddened series.
// Per acceleration trial (the hot loop), in launch groups of `batch`:
//   [resample gather -> R2C] (one batched cuFFT; with the LTO load callback
//   the resample happens inside the transform) -> k_form_norm (interbin +
//   normalise, one pass over the complex spectra) -> k_harm_peaks
//   (fractional harmonic sums + threshold + warp-aggregated compaction of
//   every (trial, fold, bin, S/N) above threshold).  Nothing per trial is
//   copied to the host; the compacted records of the whole DM come back
//   in one copy, and the host clusters (peakfinder.hpp:72-101), forms
//   frequencies and distils them (distiller.hpp).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <vector>
#include "psx_common.cuh"
#include "psx_device.cuh"
#include "psx_fft.cuh"
#include "psx_host.h"
#include "psx_stages.cuh"

namespace psx {

// Search range of each spectrum (fold 0 = the normalised interbinned
// spectrum, fold h = harmonic sum h) and the union [lo, hi).
struct PeakParams {
    int start[6];
    int end[6];
    unsigned lo, hi;
    float thresh;
};

// ------------------------------------------------------------ kernels
// Interbinned amplitude normalised with the DM's statistics
// (reference src/kernels.cu:238-259 then :496-507), for `rows` spectra.
// Two bins per thread from one 128-bit load; the previous bin of the
// pair's first element is a cached scalar load.
__global__ void __launch_bounds__(256) k_form_norm(const float* __restrict__ X, size_t xpitch,
                                                   float* __restrict__ p, size_t ppitch,
                                                   unsigned nbins, const float* __restrict__ stat)
{
    const float meanN = stat[3], stdN = stat[4];
    const float* x = X + (size_t)blockIdx.y * xpitch;
    float* o = p + (size_t)blockIdx.y * ppitch;
    const unsigned npairs = nbins / 2;
    const unsigned stride = gridDim.x * blockDim.x;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += stride) {
        const float4 v = reinterpret_cast<const float4*>(x)[q];
        float rl = 0.f, il = 0.f;
        if (q > 0) {
            rl = x[4 * q - 2];
            il = x[4 * q - 1];
        }
        float2 r;
        r.x = normalise(interbin(v.x, v.y, rl, il), meanN, stdN);
        r.y = normalise(interbin(v.z, v.w, v.x, v.y), meanN, stdN);
        reinterpret_cast<float2*>(o)[q] = r;
    }
    if ((nbins & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned k = nbins - 1;
        const float rl = k ? x[2 * k - 2] : 0.f, il = k ? x[2 * k - 1] : 0.f;
        o[k] = normalise(interbin(x[2 * k], x[2 * k + 1], rl, il), meanN, stdN);
    }
}

// Warp-aggregated append of the lanes whose `hit` is set: one atomic per
// warp and fold, records {trial, fold, bin, S/N bits}.
__device__ __forceinline__ void emit(bool hit, int trial, int fold, unsigned bin, float val,
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

__device__ __forceinline__ bool in_range(const PeakParams& pp, int h, unsigned i)
{
    return (int)i >= pp.start[h] && (int)i < pp.end[h];
}

// Fractional harmonic sums of each row with the reference's summation
// order and scales (src/kernels.cu:41-96), threshold test on the
// normalised spectrum and on every fold inside its search range, and
// compaction of the hits.  One warp covers 32 consecutive bins, so the
// gathers of fraction m/2^h touch about 32m/2^h + 1 consecutive floats.
template <int F>
__global__ void __launch_bounds__(256) k_harm_peaks(const float* __restrict__ p, size_t ppitch,
                                                    PeakParams pp, int trial0,
                                                    int4* __restrict__ rec,
                                                    unsigned* __restrict__ counter, unsigned cap)
{
    const int t = blockIdx.y;
    const int trial = trial0 + t;
    const float* __restrict__ row = p + (size_t)t * ppitch;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    const unsigned stride = gridDim.x * blockDim.x;
    const float thr = pp.thresh;
    for (unsigned base = pp.lo + warp_first; base < pp.hi; base += stride) {
        const unsigned i = base + lane;
        const bool valid = i < pp.hi;
        const unsigned ii = valid ? i : pp.hi - 1;
        float val = row[ii];
        emit(valid && in_range(pp, 0, i) && val > thr, trial, 0, i, val, rec, counter, cap, lane);
        if (F > 0) {
            val += row[frac_index<1>(ii, 1)];
            const float s = val * rsqrt(2.0);
            emit(valid && in_range(pp, 1, i) && s > thr, trial, 1, i, s, rec, counter, cap, lane);
        }
        if (F > 1) {
            val += row[frac_index<2>(ii, 3)];
            val += row[frac_index<2>(ii, 1)];
            const float s = val * 0.5;
            emit(valid && in_range(pp, 2, i) && s > thr, trial, 2, i, s, rec, counter, cap, lane);
        }
        if (F > 2) {
#pragma unroll
            for (unsigned m = 1; m < 8; m += 2) val += row[frac_index<3>(ii, m)];
            const float s = val * rsqrt(8.0);
            emit(valid && in_range(pp, 3, i) && s > thr, trial, 3, i, s, rec, counter, cap, lane);
        }
        if (F > 3) {
#pragma unroll
            for (unsigned m = 1; m < 16; m += 2) val += row[frac_index<4>(ii, m)];
            const float s = val * 0.25;
            emit(valid && in_range(pp, 4, i) && s > thr, trial, 4, i, s, rec, counter, cap, lane);
        }
        if (F > 4) {
#pragma unroll
            for (unsigned m = 1; m < 32; m += 2) val += row[frac_index<5>(ii, m)];
            const float s = val * rsqrt(32.0);
            emit(valid && in_range(pp, 5, i) && s > thr, trial, 5, i, s, rec, counter, cap, lane);
        }
    }
}

typedef void (*HarmKernel)(const float*, size_t, PeakParams, int, int4*, unsigned*, unsigned);

static HarmKernel harm_kernel(int F)
{
    switch (F) {
    case 0: return k_harm_peaks<0>;
    case 1: return k_harm_peaks<1>;
    case 2: return k_harm_peaks<2>;
    case 3: return k_harm_peaks<3>;
    case 4: return k_harm_peaks<4>;
    default: return k_harm_peaks<5>;
    }
}

}  // namespace psx

using namespace psx;

struct psx_search {
    psx_search_config cfg{};
    std::vector<float> bf, bw;
    size_t N = 0, B = 0, Bp = 0;
    int F = 0;
    int batch = 1;
    int device = 0;
    cudaStream_t st = nullptr;
    bool own_stream = false;
    double bin_width = 0.0;
    float bin_width_f = 0.f;
    float tobs = 0.f;
    PeakParams pk{};
    float factor[6] = {0, 0, 0, 0, 0, 0};

    float* d_tim = nullptr;
    float* d_tr = nullptr;
    float* d_X = nullptr;
    float* d_p = nullptr;
    void* d_med = nullptr;
    double2* d_part = nullptr;
    double* d_sums = nullptr;
    float* d_stat = nullptr;
    float* d_mean = nullptr;
    float* d_bf = nullptr;
    float* d_bw = nullptr;
    double* d_ktab = nullptr;
    double* d_kbatch = nullptr;
    size_t ktab_cap = 0;
    double* h_ktab = nullptr;
    int4* d_rec = nullptr;
    unsigned* d_count = nullptr;
    size_t rec_cap = 0;
    int4* h_rec = nullptr;
    unsigned* h_count = nullptr;

    FftPlan r2c1, c2r1;
    std::map<int, FftPlan*> r2cb;
    std::map<int, cudaGraphExec_t> graphs;
    struct GraphCounts {
        int launches, ffts, groups;
    };
    std::map<int, GraphCounts> graph_counts;

    std::vector<float> accs;
    psx_search_info info{};
    int launches = 0;
    int ffts = 0;

    ~psx_search() { release(); }

    void release()
    {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second);
        graphs.clear();
        for (auto& p : r2cb) delete p.second;
        r2cb.clear();
        r2c1.destroy();
        c2r1.destroy();
        void* dev[] = {d_tim, d_tr, d_X, d_p, d_med, d_part, d_sums, d_stat, d_mean,
                       d_bf, d_bw, d_ktab, d_kbatch, d_rec, d_count};
        for (void* q : dev)
            if (q) cudaFree(q);
        d_tim = d_tr = d_X = d_p = nullptr;
        d_med = nullptr;
        d_part = nullptr;
        d_sums = nullptr;
        d_stat = d_mean = d_bf = d_bw = nullptr;
        d_ktab = d_kbatch = nullptr;
        d_rec = nullptr;
        d_count = nullptr;
        if (h_ktab) cudaFreeHost(h_ktab);
        if (h_rec) cudaFreeHost(h_rec);
        if (h_count) cudaFreeHost(h_count);
        h_ktab = nullptr;
        h_rec = nullptr;
        h_count = nullptr;
        if (own_stream && st) cudaStreamDestroy(st);
        st = nullptr;
        own_stream = false;
    }

    bool batched() const { return cfg.mode == PSX_MODE_BATCHED; }
    bool callback() const { return batched() && cfg.use_fft_callback; }

    int get_plan(int b, FftPlan** out);
    int grow_records(size_t need);
    int grow_ktab(size_t need);
    int prologue(const float* series, size_t nsamps, bool on_device);
    int trials_enqueue(int nacc);
    int run_trials(int nacc);
    int collect(float dm, int dm_idx, int output, std::vector<psx_candidate>& out,
                std::vector<int>& nassoc, std::vector<int>& trial_of);
};

static size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

static int default_batch(size_t n)
{
    size_t b = ((size_t)1 << 26) / n;
    if (b < 1) b = 1;
    if (b > 64) b = 64;
    size_t p = 1;
    while (p * 2 <= b) p *= 2;
    return (int)p;
}

int psx_search::get_plan(int b, FftPlan** out)
{
    auto it = r2cb.find(b);
    if (it != r2cb.end()) {
        *out = it->second;
        return PSX_OK;
    }
    FftPlan* p = new (std::nothrow) FftPlan;
    if (!p) return PSX_ERR_ALLOC;
    int rc = p->create(N, b, PSX_FFT_R2C, N, Bp, callback());
    if (rc == PSX_OK && callback()) rc = p->set_resample(d_tim, d_kbatch, st);
    if (rc != PSX_OK) {
        delete p;
        return rc;
    }
    r2cb[b] = p;
    *out = p;
    return PSX_OK;
}

int psx_search::grow_records(size_t need)
{
    if (need <= rec_cap) return PSX_OK;
    size_t cap = round_up(need + need / 4, 4096);
    if (d_rec) cudaFree(d_rec);
    if (h_rec) cudaFreeHost(h_rec);
    d_rec = nullptr;
    h_rec = nullptr;
    rec_cap = 0;
    PSX_CUDA(cudaMalloc(&d_rec, sizeof(int4) * cap));
    PSX_CUDA(cudaMallocHost(&h_rec, sizeof(int4) * cap));
    rec_cap = cap;
    // captured schedules hold the old buffer
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    graphs.clear();
    return PSX_OK;
}

int psx_search::grow_ktab(size_t need)
{
    if (need <= ktab_cap) return PSX_OK;
    size_t cap = round_up(need + need / 2, 256);
    PSX_CUDA(cudaStreamSynchronize(st));
    if (d_ktab) cudaFree(d_ktab);
    if (h_ktab) cudaFreeHost(h_ktab);
    d_ktab = nullptr;
    h_ktab = nullptr;
    ktab_cap = 0;
    PSX_CUDA(cudaMalloc(&d_ktab, sizeof(double) * cap));
    PSX_CUDA(cudaMallocHost(&h_ktab, sizeof(double) * cap));
    ktab_cap = cap;
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    graphs.clear();
    return PSX_OK;
}

// src/pipeline_multi.cu:170-238 for one series.
int psx_search::prologue(const float* series, size_t nsamps, bool on_device)
{
    const size_t ncopy = std::min(nsamps, N);
    PSX_CUDA(cudaMemcpyAsync(d_tim, series, sizeof(float) * ncopy,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    // baseline removal over the copied samples (timeseries.hpp:282-287,
    // src/kernels.cu:463-479)
    int count = 0;
    float mean = 0.f;
    do {
        PSX_TRY(remove_baseline_pass(d_tim, ncopy, d_part, d_sums, d_mean, st));
        launches += 4;
        PSX_CUDA(cudaMemcpyAsync(h_count + 2, d_mean, sizeof(float), cudaMemcpyDeviceToHost, st));
        PSX_CUDA(cudaStreamSynchronize(st));
        std::memcpy(&mean, h_count + 2, sizeof(float));
        if (count++ > 100) break;
    } while (std::fabs(mean) > 5e-7 * (double)ncopy);
    // zero padding (pipeline_multi.cu:179-187)
    if (ncopy < N) {
        PSX_TRY(launch_fill(d_tim + ncopy, N - ncopy, 0.f, st));
        ++launches;
    }
    PSX_TRY(r2c1.exec(d_tim, d_X, st));
    ++ffts;
    // amplitude spectrum into the first row of d_p (spectrumformer.hpp:16-22)
    PSX_TRY(psx_form_power_series(d_X, d_p, B, 0, reinterpret_cast<psx_stream_t>(st)));
    ++launches;
    // running median and division (dereddener.hpp:41-66)
    PSX_TRY(launch_running_median(d_p, B, bin_width, cfg.boundary_5_freq, cfg.boundary_25_freq,
                                  nullptr, d_X, d_med, st));
    launches += 4;
    if (!bf.empty()) {
        PSX_TRY(launch_zap(d_X, d_bf, d_bw, bin_width_f, bf.size(), B, st));
        ++launches;
    }
    // interbin statistics (pipeline_multi.cu:230-234) -> mean*N, std*N
    PSX_TRY(launch_stats(d_X, true, 0, B, d_part, d_sums, d_stat, (float)N, st));
    launches += 2;
    PSX_TRY(c2r1.exec(d_X, d_tim, st));
    ++ffts;
    return PSX_OK;
}

// Enqueues every acceleration trial of the DM (k factors already in
// d_ktab) plus the reset of the record counter.
int psx_search::trials_enqueue(int nacc)
{
    PSX_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned) * 2, st));
    const unsigned T = 256;
    HarmKernel hk = harm_kernel(F);
    const unsigned span = pk.hi > pk.lo ? pk.hi - pk.lo : 0;
    int t0 = 0, groups = 0;
    while (t0 < nacc) {
        int b = 1;
        const float* xin = d_tr;
        if (batched()) {
            b = batch;
            while (b > nacc - t0) b >>= 1;
            FftPlan* plan = nullptr;
            PSX_TRY(get_plan(b, &plan));
            if (callback()) {
                PSX_CUDA(cudaMemcpyAsync(d_kbatch, d_ktab + t0, sizeof(double) * b,
                                         cudaMemcpyDeviceToDevice, st));
            } else {
                PSX_TRY(launch_resample(d_tim, d_tr, N, d_ktab + t0, 0.0, b, N, false, st));
                ++launches;
            }
            PSX_TRY(plan->exec(xin, d_X, st));
            ++ffts;
        } else {
            PSX_TRY(launch_resample(d_tim, d_tr, N, d_ktab + t0, 0.0, 1, N, false, st));
            ++launches;
            PSX_TRY(r2c1.exec(d_tr, d_X, st));
            ++ffts;
        }
        dim3 gf(grid_for(B / 2 + 1, T, 4), (unsigned)b);
        k_form_norm<<<gf, T, 0, st>>>(d_X, 2 * Bp, d_p, Bp, (unsigned)B, d_stat);
        ++launches;
        if (span) {
            dim3 gh(grid_for(span, T, 8), (unsigned)b);
            hk<<<gh, T, 0, st>>>(d_p, Bp, pk, t0, d_rec, d_count, (unsigned)rec_cap);
            ++launches;
        }
        PSX_TRY(launch_status("search trial kernels"));
        t0 += b;
        ++groups;
    }
    info.nbatches = groups;
    return PSX_OK;
}

int psx_search::run_trials(int nacc)
{
    const bool graph = batched() && cfg.use_graph;
    info.graph = 0;
    if (!graph) return trials_enqueue(nacc);
    auto it = graphs.find(nacc);
    if (it == graphs.end()) {
        // plans must exist before capture (creation allocates and syncs)
        for (int b = batch; b >= 1; b >>= 1) {
            FftPlan* p = nullptr;
            PSX_TRY(get_plan(b, &p));
        }
        PSX_CUDA(cudaStreamSynchronize(st));
        const int l0 = launches, f0 = ffts;
        PSX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = trials_enqueue(nacc);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc != PSX_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        PSX_CUDA(e);
        cudaGraphExec_t ge = nullptr;
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        PSX_CUDA(e);
        it = graphs.emplace(nacc, ge).first;
        // the captured work is counted at every replay below
        graph_counts[nacc] = GraphCounts{launches - l0, ffts - f0, info.nbatches};
        launches = l0;
        ffts = f0;
    }
    PSX_CUDA(cudaGraphLaunch(it->second, st));
    const GraphCounts& gc = graph_counts[nacc];
    launches += gc.launches;
    ffts += gc.ffts;
    info.nbatches = gc.groups;
    info.graph = 1;
    return PSX_OK;
}

// Host side of one DM: record copy-back, clustering per (trial, fold),
// candidate frequencies, per-trial harmonic distillation and optionally
// the per-DM acceleration distillation (pipeline_multi.cu:283-294).
int psx_search::collect(float dm, int dm_idx, int output, std::vector<psx_candidate>& out,
                        std::vector<int>& nassoc, std::vector<int>& trial_of)
{
    const size_t nrec = h_count[0];
    if (nrec) {
        PSX_CUDA(cudaMemcpyAsync(h_rec, d_rec, sizeof(int4) * nrec, cudaMemcpyDeviceToHost, st));
        PSX_CUDA(cudaStreamSynchronize(st));
    }
    // order by (trial, fold, bin): the bins of one spectrum ascending, as
    // the reference's order-preserving copy_if leaves them
    std::sort(h_rec, h_rec + nrec, [](const int4& a, const int4& b) {
        if (a.x != b.x) return a.x < b.x;
        if (a.y != b.y) return a.y < b.y;
        return a.z < b.z;
    });
    out.clear();
    nassoc.clear();
    trial_of.clear();
    std::vector<int> idx, pidx;
    std::vector<float> snr, psnr;
    std::vector<psx_candidate> tc;
    size_t r = 0;
    const int nacc = (int)accs.size();
    for (int t = 0; t < nacc; ++t) {
        tc.clear();
        for (int h = 0; h <= F; ++h) {
            idx.clear();
            snr.clear();
            while (r < nrec && h_rec[r].x == t && h_rec[r].y == h) {
                idx.push_back(h_rec[r].z);
                float v;
                std::memcpy(&v, &h_rec[r].w, sizeof v);
                snr.push_back(v);
                ++r;
            }
            if (idx.empty()) continue;
            pidx.resize(idx.size());
            psnr.resize(idx.size());
            const size_t np = unique_peaks(idx.data(), snr.data(), idx.size(), cfg.min_gap,
                                           pidx.data(), psnr.data());
            for (size_t k = 0; k < np; ++k)
                tc.push_back(psx_candidate{dm, dm_idx, accs[t], h, psnr[k],
                                           (float)pidx[k] * factor[h]});
        }
        // skip records of folds that were not consumed (cannot happen for
        // folds 0..F, kept for robustness)
        while (r < nrec && h_rec[r].x == t) ++r;
        if (tc.empty()) continue;
        const size_t keep = distill(PSX_DISTILL_HARMONIC, tc.data(), tc.size(), cfg.freq_tol,
                                    cfg.max_harm, tobs, 0, 1, nullptr);
        for (size_t k = 0; k < keep; ++k) {
            out.push_back(tc[k]);
            trial_of.push_back(t);
        }
    }
    if (output == PSX_OUT_DM && !out.empty()) {
        // The acceleration distiller reorders candidates; carry the trial
        // index through it by tagging the S/N-sorted order afterwards.
        std::vector<psx_candidate> c = out;
        nassoc.assign(c.size(), 0);
        const size_t keep = distill(PSX_DISTILL_ACCEL, c.data(), c.size(), cfg.freq_tol,
                                    cfg.max_harm, tobs, 1, 1, nassoc.data());
        c.resize(keep);
        nassoc.resize(keep);
        // trial index of each survivor: its acceleration's position in the list
        trial_of.assign(keep, -1);
        for (size_t k = 0; k < keep; ++k) {
            auto it = std::lower_bound(accs.begin(), accs.end(), c[k].acc);
            if (it != accs.end() && *it == c[k].acc) trial_of[k] = (int)(it - accs.begin());
        }
        out.swap(c);
    } else {
        nassoc.assign(out.size(), 0);
    }
    return PSX_OK;
}

extern "C" {

void psx_search_config_defaults(psx_search_config* c, size_t fft_size, float tsamp)
{
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->fft_size = fft_size;
    c->tsamp = tsamp;
    c->cdm = 0.0f;
    c->acc_lo = 0.0f;
    c->acc_hi = 0.0f;
    c->acc_tol = 1.10f;
    c->acc_pulse_width = 64e-6f;
    c->cfreq_hz = 1475.12e6f;
    c->ch_bw_hz = 1.09e6f;
    c->nharmonics = 4;
    c->min_snr = 9.0f;
    c->min_freq = 0.1f;
    c->max_freq = 1100.0f;
    c->min_gap = 30;
    c->freq_tol = 0.0001f;
    c->max_harm = 16.0f;
    c->boundary_5_freq = 0.05f;
    c->boundary_25_freq = 0.5f;
    c->mode = PSX_MODE_BATCHED;
    c->batch = 0;
    c->use_fft_callback = 1;
    c->use_graph = 1;
}

static int check_config(const psx_search_config* c)
{
    if (!c) {
        set_error("search: null config");
        return PSX_ERR_INVALID;
    }
    if (!fft_size_supported(c->fft_size) || c->fft_size < 1024 || c->fft_size > ((size_t)1 << 28)) {
        set_error("search: fft_size %zu must be 2^k or 3*2^k within [1024, 2^28]", c->fft_size);
        return PSX_ERR_INVALID;
    }
    if (!(c->tsamp > 0.f)) {
        set_error("search: tsamp must be positive");
        return PSX_ERR_INVALID;
    }
    if (c->nharmonics < 0 || c->nharmonics > 5) {
        set_error("search: nharmonics must be 0..5 (the reference sums at most 5 folds)");
        return PSX_ERR_INVALID;
    }
    if (c->mode != PSX_MODE_PLAIN && c->mode != PSX_MODE_BATCHED) {
        set_error("search: unknown mode %d", c->mode);
        return PSX_ERR_INVALID;
    }
    if (c->batch < 0 || c->batch > 1024) {
        set_error("search: batch must be 0..1024");
        return PSX_ERR_INVALID;
    }
    if (c->nbirdies && (!c->birdie_freqs || !c->birdie_widths)) {
        set_error("search: birdie arrays missing");
        return PSX_ERR_INVALID;
    }
    if (c->acc_hi < c->acc_lo) {
        set_error("search: acc_hi < acc_lo");
        return PSX_ERR_INVALID;
    }
    return PSX_OK;
}

static int effective_batch(const psx_search_config* c)
{
    if (c->mode != PSX_MODE_BATCHED) return 1;
    int b = c->batch ? c->batch : default_batch(c->fft_size);
    int p = 1;
    while (p * 2 <= b) p *= 2;
    return p;
}

size_t psx_search_footprint(const psx_search_config* c)
{
    if (check_config(c) != PSX_OK) return 0;
    const size_t N = c->fft_size, B = N / 2 + 1, Bp = round_up(B, 64);
    const size_t b = (size_t)effective_batch(c);
    const bool cb = c->mode == PSX_MODE_BATCHED && c->use_fft_callback;
    size_t bytes = 0;
    bytes += sizeof(float) * N;                       // resident dereddened series
    bytes += sizeof(float) * N * (cb ? 1 : b);        // resampled series
    bytes += sizeof(float) * 2 * Bp * b;              // complex spectra
    bytes += sizeof(float) * Bp * b;                  // normalised spectra
    bytes += median_scratch_bytes(B);
    bytes += sizeof(int4) * ((size_t)1 << 20);        // initial record buffer
    // cuFFT work areas: about one transform's worth per batched plan size
    bytes += sizeof(float) * 2 * Bp * (2 * b + 2);
    return bytes;
}

int psx_search_create(const psx_search_config* cfg, psx_search** out)
{
    clear_error();
    if (!out) return PSX_ERR_INVALID;
    *out = nullptr;
    PSX_TRY(check_config(cfg));
    psx_search* s = new (std::nothrow) psx_search;
    if (!s) return PSX_ERR_ALLOC;
    s->cfg = *cfg;
    if (cfg->nbirdies) {
        s->bf.assign(cfg->birdie_freqs, cfg->birdie_freqs + cfg->nbirdies);
        s->bw.assign(cfg->birdie_widths, cfg->birdie_widths + cfg->nbirdies);
    }
    s->cfg.birdie_freqs = nullptr;
    s->cfg.birdie_widths = nullptr;
    s->N = cfg->fft_size;
    s->B = s->N / 2 + 1;
    s->Bp = round_up(s->B, 64);
    s->F = cfg->nharmonics;
    s->batch = effective_batch(cfg);
    // pipeline_multi.cu:126-128: tobs and bin width are floats
    s->tobs = (float)s->N * cfg->tsamp;
    s->bin_width_f = (float)(1.0 / (double)s->tobs);
    s->bin_width = (double)s->bin_width_f;
    // search ranges of every fold (peakfinder.hpp:123-128)
    unsigned lo = 0xffffffffu, hi = 0;
    for (int h = 0; h <= 5; ++h) {
        int st, en;
        float fac;
        peak_range((unsigned)s->B, s->bin_width, h, cfg->min_freq, cfg->max_freq, &st, &en, &fac);
        if (st < 0) st = 0;
        if (en > (int)s->B) en = (int)s->B;
        if (h > s->F) {
            st = 0;
            en = 0;
        }
        s->pk.start[h] = st;
        s->pk.end[h] = en;
        s->factor[h] = fac;
        if (en > st) {
            lo = std::min(lo, (unsigned)st);
            hi = std::max(hi, (unsigned)en);
        }
    }
    s->pk.lo = hi > lo ? lo : 0;
    s->pk.hi = hi > lo ? hi : 0;
    s->pk.thresh = cfg->min_snr;

    int rc = PSX_OK;
    auto fail = [&](int code) {
        delete s;
        return code;
    };
    if ((rc = cuda_status(cudaGetDevice(&s->device), "cudaGetDevice")) != PSX_OK) return fail(rc);
    if ((rc = cuda_status(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking),
                          "cudaStreamCreate")) != PSX_OK)
        return fail(rc);
    s->own_stream = true;
    const size_t N = s->N, Bp = s->Bp;
    const size_t b = (size_t)s->batch;
    const bool cb = s->callback();
    const int nb = reduction_blocks();
#define ALLOC(ptr, bytes)                                                        \
    if ((rc = cuda_status(cudaMalloc((void**)&(ptr), (bytes)), "cudaMalloc")) != \
        PSX_OK)                                                                  \
        return fail(rc == PSX_ERR_CUDA ? PSX_ERR_ALLOC : rc);
    ALLOC(s->d_tim, sizeof(float) * N);
    ALLOC(s->d_tr, sizeof(float) * N * (cb ? 1 : b));
    ALLOC(s->d_X, sizeof(float) * 2 * Bp * b);
    ALLOC(s->d_p, sizeof(float) * Bp * b);
    ALLOC(s->d_med, median_scratch_bytes(s->B));
    ALLOC(s->d_part, sizeof(double2) * nb);
    ALLOC(s->d_sums, sizeof(double) * 2);
    ALLOC(s->d_stat, sizeof(float) * 8);
    ALLOC(s->d_mean, sizeof(float) * 2);
    ALLOC(s->d_kbatch, sizeof(double) * b);
    ALLOC(s->d_count, sizeof(unsigned) * 2);
    if (!s->bf.empty()) {
        ALLOC(s->d_bf, sizeof(float) * s->bf.size());
        ALLOC(s->d_bw, sizeof(float) * s->bw.size());
    }
#undef ALLOC
    if ((rc = cuda_status(cudaMallocHost(&s->h_count, sizeof(unsigned) * 4), "cudaMallocHost")) !=
        PSX_OK)
        return fail(PSX_ERR_ALLOC);
    if (!s->bf.empty()) {
        cudaMemcpy(s->d_bf, s->bf.data(), sizeof(float) * s->bf.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(s->d_bw, s->bw.data(), sizeof(float) * s->bw.size(), cudaMemcpyHostToDevice);
    }
    // zero the padded tails once so no uninitialised memory is ever read
    cudaMemsetAsync(s->d_X, 0, sizeof(float) * 2 * Bp * b, s->st);
    cudaMemsetAsync(s->d_p, 0, sizeof(float) * Bp * b, s->st);
    cudaMemsetAsync(s->d_kbatch, 0, sizeof(double) * b, s->st);
    if ((rc = s->grow_records((size_t)1 << 20)) != PSX_OK) return fail(rc);
    if ((rc = s->grow_ktab(1024)) != PSX_OK) return fail(rc);
    if ((rc = s->r2c1.create(N, 1, PSX_FFT_R2C, 0, 0, false)) != PSX_OK) return fail(rc);
    if ((rc = s->c2r1.create(N, 1, PSX_FFT_C2R, 0, 0, false)) != PSX_OK) return fail(rc);
    if (s->batched()) {
        FftPlan* p = nullptr;
        if ((rc = s->get_plan(s->batch, &p)) != PSX_OK) return fail(rc);
    }
    if ((rc = cuda_status(cudaStreamSynchronize(s->st), "search create")) != PSX_OK)
        return fail(rc);
    s->info.batch = s->batch;
    s->info.fft_callback = cb ? 1 : 0;
    *out = s;
    return PSX_OK;
}

int psx_search_destroy(psx_search* s)
{
    clear_error();
    if (!s) return PSX_OK;
    if (s->st) cudaStreamSynchronize(s->st);
    delete s;
    return PSX_OK;
}

int psx_search_set_stream(psx_search* s, psx_stream_t stream)
{
    clear_error();
    if (!s) return PSX_ERR_INVALID;
    PSX_CUDA(cudaStreamSynchronize(s->st));
    if (s->own_stream) cudaStreamDestroy(s->st);
    s->own_stream = false;
    s->st = cs(stream);
    // graphs are stream independent; nothing else holds the stream
    return PSX_OK;
}

int psx_search_dm(psx_search* s, const float* series, size_t nsamps, int series_on_device,
                  float dm, int dm_idx, int output, psx_candidate* h_out, int* h_nassoc,
                  int* h_trial, size_t cap, size_t* n_out)
{
    clear_error();
    if (!s || !series || !n_out || nsamps == 0 || (output != PSX_OUT_TRIAL && output != PSX_OUT_DM)) {
        set_error("search_dm: bad arguments");
        return PSX_ERR_INVALID;
    }
    *n_out = 0;
    s->launches = 0;
    s->ffts = 0;
    const int dev_rc = cuda_status(cudaSetDevice(s->device), "cudaSetDevice");
    if (dev_rc != PSX_OK) return dev_rc;
    PSX_TRY(s->prologue(series, nsamps, series_on_device != 0));
    const psx_search_config& c = s->cfg;
    s->accs = accel_list(c.acc_lo, c.acc_hi, c.acc_tol, c.acc_pulse_width, s->N, c.tsamp,
                         c.cfreq_hz, c.ch_bw_hz, dm, c.cdm);
    const int nacc = (int)s->accs.size();
    PSX_TRY(s->grow_ktab((size_t)nacc));
    for (int t = 0; t < nacc; ++t) s->h_ktab[t] = accel_fact(s->accs[t], c.tsamp);
    PSX_CUDA(cudaMemcpyAsync(s->d_ktab, s->h_ktab, sizeof(double) * nacc, cudaMemcpyHostToDevice,
                             s->st));
    for (int attempt = 0; attempt < 2; ++attempt) {
        PSX_TRY(s->run_trials(nacc));
        PSX_CUDA(cudaMemcpyAsync(s->h_count, s->d_count, sizeof(unsigned) * 2,
                                 cudaMemcpyDeviceToHost, s->st));
        PSX_CUDA(cudaStreamSynchronize(s->st));
        if (s->h_count[0] <= s->rec_cap) break;
        // more hits than the record buffer holds: grow it and run again
        PSX_TRY(s->grow_records(s->h_count[0]));
        if (attempt == 1) {
            set_error("search_dm: record buffer overflow");
            return PSX_ERR_OVERFLOW;
        }
    }
    s->info.ntrials = nacc;
    s->info.above_threshold = (long long)s->h_count[0];
    std::vector<psx_candidate> out;
    std::vector<int> nassoc, trial_of;
    PSX_TRY(s->collect(dm, dm_idx, output, out, nassoc, trial_of));
    s->info.kernel_launches = s->launches;
    s->info.fft_launches = s->ffts;
    *n_out = out.size();
    if (out.size() > cap || (!h_out && out.size())) {
        set_error("search_dm: %zu candidates, buffer holds %zu", out.size(), cap);
        return PSX_ERR_OVERFLOW;
    }
    if (!out.empty()) std::memcpy(h_out, out.data(), sizeof(psx_candidate) * out.size());
    for (size_t k = 0; k < out.size(); ++k) {
        if (h_nassoc) h_nassoc[k] = nassoc[k];
        if (h_trial) h_trial[k] = trial_of[k];
    }
    return PSX_OK;
}

int psx_search_last_info(const psx_search* s, psx_search_info* info)
{
    if (!s || !info) return PSX_ERR_INVALID;
    *info = s->info;
    return PSX_OK;
}

int psx_search_debug_tap(psx_search* s, int trial, float* h_tim_dered, float* h_tim_r,
                         float* h_pspec, float* h_norm2)
{
    clear_error();
    if (!s) return PSX_ERR_INVALID;
    if (h_tim_dered)
        PSX_CUDA(cudaMemcpyAsync(h_tim_dered, s->d_tim, sizeof(float) * s->N,
                                 cudaMemcpyDeviceToHost, s->st));
    if (h_norm2)
        PSX_CUDA(cudaMemcpyAsync(h_norm2, s->d_stat + 3, sizeof(float) * 2, cudaMemcpyDeviceToHost,
                                 s->st));
    if (h_tim_r || h_pspec) {
        if (trial < 0 || trial >= (int)s->accs.size()) {
            set_error("debug_tap: trial %d out of range", trial);
            return PSX_ERR_INVALID;
        }
        PSX_TRY(launch_resample(s->d_tim, s->d_tr, s->N, nullptr,
                                accel_fact(s->accs[trial], s->cfg.tsamp), 1, s->N, false, s->st));
        if (h_tim_r)
            PSX_CUDA(cudaMemcpyAsync(h_tim_r, s->d_tr, sizeof(float) * s->N,
                                     cudaMemcpyDeviceToHost, s->st));
        if (h_pspec) {
            PSX_TRY(s->r2c1.exec(s->d_tr, s->d_X, s->st));
            dim3 gf(grid_for(s->B / 2 + 1, 256, 4), 1);
            k_form_norm<<<gf, 256, 0, s->st>>>(s->d_X, 2 * s->Bp, s->d_p, s->Bp, (unsigned)s->B,
                                               s->d_stat);
            PSX_TRY(launch_status("debug tap"));
            PSX_CUDA(cudaMemcpyAsync(h_pspec, s->d_p, sizeof(float) * s->B,
                                     cudaMemcpyDeviceToHost, s->st));
        }
    }
    return cuda_status(cudaStreamSynchronize(s->st), "debug tap");
}

}  // extern "C"
