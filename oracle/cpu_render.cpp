/*
 * cpu_render.cpp -- an FP32 CPU rendering of the per-DM acceleration
 * search (src/pipeline_multi.cu:161-290), the reported CPU baseline of the
 * benchmark.  TEST INFRASTRUCTURE ONLY: only bench.py's cpu_baseline leg
 * and tests/ load it; the product never does.
 *
 * FFTW is not in this image, so the transforms are libtorch's CPU FFT
 * (at::fft_rfft / at::fft_irfft, backed by Intel MKL in this build).
 *
 *   per DM trial (once): baseline removal, zero padding, R2C, amplitudes,
 *     running median, dereddening, zapping, interbinned statistics, C2R --
 *     in double precision with the oracle's stage functions (psx_oracle.c)
 *     and MKL's double-precision transforms;
 *   per acceleration trial (the hot loop), in FP32, trials spread over
 *     `nthreads` worker threads with single-threaded transforms:
 *     resampleII through the reference's FP64 index (src/kernels.cu:
 *     321-324, fused multiply-add as the reference compiles it), MKL's
 *     real transform, interbinning (src/kernels.cu:238-259), normalisation
 *     (src/kernels.cu:496-507), the fractional harmonic sums in the
 *     reference's order (src/kernels.cu:34-100) fused with the threshold
 *     test of every fold, peak clustering and the frequencies of
 *     include/transforms/peakfinder.hpp:72-94, and the per-trial harmonic
 *     distillation (include/transforms/distiller.hpp:63-108).
 */
#include <ATen/ATen.h>
#include <ATen/Parallel.h>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>
#include "psx_oracle.h"

namespace {

struct Hit {
    int idx;
    double snr;
};

/* One acceleration trial in FP32; appends its harmonic-distilled
   candidates to `out`. */
void search_trial(const float* tim, size_t N, float acc, const orc_search_params* p, float meanN,
                  float sdN, double bw, at::Tensor& tim_rt, at::Tensor& X,
                  std::vector<float>& pspec, std::vector<std::vector<Hit>>& hits,
                  std::vector<orc_candidate>& out)
{
    const size_t B = N / 2 + 1;
    const int F = p->nharmonics;
    // resampleII: out[i] = in[rn(fma(i k, i - N, i))] (src/kernels.cu:321-324, 361)
    const double k = orc_accel_fact(acc, p->tsamp), size = (double)N;
    float* tim_r = tim_rt.data_ptr<float>();
    for (size_t i = 0; i < N; ++i) {
        const double id = (double)i;
        const double v = std::fma(id * k, id - size, id);
        const double r = std::nearbyint(v);
        const size_t j = v > 0.0 ? (size_t)r : 0;
        tim_r[i] = j < N ? tim[j] : 0.0f;
    }
    at::fft_rfft_out(X, tim_rt);
    const float* xc = reinterpret_cast<const float*>(X.data_ptr());
    // interbin + normalise
    float pre = 0.f, pim = 0.f;
    for (size_t i = 0; i < B; ++i) {
        const float re = xc[2 * i], im = xc[2 * i + 1];
        const float dr = re - pre, di = im - pim;
        const float a = std::sqrt(std::fmax(re * re + im * im, 0.5f * (dr * dr + di * di)));
        pspec[i] = (a - meanN) / sdN;
        pre = re;
        pim = im;
    }
    // harmonic sums fused with every fold's threshold test (bins ascending)
    int start[6], end[6];
    float factor[6];
    for (int h = 0; h <= F; ++h) {
        orc_peak_range((unsigned)B, bw, h, p->min_freq, p->max_freq, &start[h], &end[h],
                       &factor[h]);
        if (start[h] < 0) start[h] = 0;
        hits[h].clear();
    }
    static const double scale[6] = {1.0, 0.70710678118654752440, 0.5, 0.35355339059327376220,
                                    0.25, 0.17677669529663688110};
    const float thr = p->min_snr;
    const float* in0 = pspec.data();
    for (size_t i = 0; i < B; ++i) {
        float val = in0[i];
        if (val > thr && (int)i >= start[0] && (int)i < end[0]) hits[0].push_back({(int)i, val});
        for (int h = 1; h <= F; ++h) {
            const size_t half = (size_t)1 << (h - 1);
            if (h == 2) {
                val += in0[(i * 3 + half) >> h];
                val += in0[(i + half) >> h];
            } else {
                for (size_t m = 1; m < 2 * half; m += 2) val += in0[(i * m + half) >> h];
            }
            const float s = (float)((double)val * scale[h]);
            if (s > thr && (int)i >= start[h] && (int)i < end[h]) hits[h].push_back({(int)i, s});
        }
    }
    // clustering and frequencies, then the trial's harmonic distillation
    std::vector<orc_candidate> tc;
    std::vector<int> ai, pi;
    std::vector<double> as, ps;
    for (int h = 0; h <= F; ++h) {
        const size_t n = hits[h].size();
        ai.resize(n);
        as.resize(n);
        for (size_t q = 0; q < n; ++q) {
            ai[q] = hits[h][q].idx;
            as[q] = hits[h][q].snr;
        }
        pi.resize(n + 1);
        ps.resize(n + 1);
        const size_t np = orc_identify_unique_peaks(ai.data(), as.data(), n, p->min_gap,
                                                    pi.data(), ps.data());
        for (size_t q = 0; q < np; ++q)
            tc.push_back(orc_candidate{p->dm, p->dm_idx, acc, h, (float)ps[q],
                                       (float)pi[q] * factor[h]});
    }
    std::vector<int> keep(tc.size());
    orc_harmonic_distill(tc.data(), tc.size(), p->freq_tol, p->max_harm, 1, keep.data(),
                         nullptr);
    for (size_t q = 0; q < tc.size(); ++q)
        if (keep[q]) out.push_back(tc[q]);
}

}  // namespace

extern "C" {

/* One DM trial: every acceleration trial's harmonic-distilled candidates
   in trial order (trial_of[i] = trial index), like orc_search_dm.  Returns
   the count, or (size_t)-1 on bad arguments or when cap is too small;
   *seconds = wall time of the whole DM trial (prologue included). */
size_t cpu_search_dm(const float* series, size_t nsamps, const orc_search_params* p,
                     int nthreads, orc_candidate* out, int* trial_of, size_t cap,
                     double* seconds)
{
    const size_t N = p->fft_size, B = N / 2 + 1;
    if (p->nharmonics < 0 || p->nharmonics > 5 || N < 16 || nthreads < 1) return (size_t)-1;
    at::set_num_threads(1);
    const auto t0 = std::chrono::steady_clock::now();
    // ---- prologue (double precision)
    std::vector<double> tim(N, 0.0), pspec(B), med(B);
    const size_t ncopy = std::min(nsamps, N);
    for (size_t i = 0; i < ncopy; ++i) tim[i] = series[i];
    orc_remove_baseline(tim.data(), ncopy);
    const float tobs = (float)N * p->tsamp;
    const double bw = (float)(1.0 / (double)tobs);
    at::Tensor Xd = at::fft_rfft(at::from_blob(tim.data(), {(int64_t)N}, at::kDouble));
    double* X = reinterpret_cast<double*>(Xd.data_ptr());
    orc_form_power(X, B, pspec.data());
    orc_running_median(pspec.data(), B, bw, 0.05f, 0.5f, med.data());
    orc_deredden(X, med.data(), B);
    if (p->nbirdies)
        orc_zap(X, B, (float)bw, p->birdie_freqs, p->birdie_widths, p->nbirdies);
    orc_form_interbin(X, B, pspec.data());
    double mean, rms, sd;
    orc_stats(pspec.data(), B, 0, &mean, &rms, &sd);
    at::Tensor td = at::fft_irfft(Xd, (int64_t)N, -1, "forward");  // unnormalised inverse
    std::vector<float> timf(N);
    const double* tdp = td.data_ptr<double>();
    for (size_t i = 0; i < N; ++i) timf[i] = (float)tdp[i];
    const float meanN = (float)(mean * (double)N), sdN = (float)(sd * (double)N);
    // ---- acceleration trials (FP32), spread over the workers
    size_t nacc = orc_accel_list(p->acc_lo, p->acc_hi, p->acc_tol, p->acc_pulse_width, N,
                                 p->tsamp, p->cfreq, p->ch_bw, p->dm, p->cdm, nullptr, 0);
    std::vector<float> accs(nacc + 1);
    nacc = orc_accel_list(p->acc_lo, p->acc_hi, p->acc_tol, p->acc_pulse_width, N, p->tsamp,
                          p->cfreq, p->ch_bw, p->dm, p->cdm, accs.data(), accs.size());
    std::vector<std::vector<orc_candidate>> per_trial(nacc);
    std::atomic<size_t> next{0};
    auto work = [&]() {
        // the intra-op thread count is a per-thread setting (OpenMP):
        // every worker runs its transforms on itself alone
        at::set_num_threads(1);
        // torch's allocations are 64-byte aligned: the transform then takes
        // the same code path in every worker, so results do not depend on
        // which thread ran a trial
        at::Tensor tim_r = at::empty({(int64_t)N}, at::kFloat);
        std::vector<float> ps(B);
        at::Tensor Xt = at::empty({(int64_t)B}, at::kComplexFloat);
        std::vector<std::vector<Hit>> hits(6);
        for (;;) {
            const size_t t = next.fetch_add(1);
            if (t >= nacc) break;
            search_trial(timf.data(), N, accs[t], p, meanN, sdN, bw, tim_r, Xt, ps, hits,
                         per_trial[t]);
        }
    };
    const int nt = (int)std::min<size_t>((size_t)nthreads, std::max<size_t>(nacc, 1));
    std::vector<std::thread> pool;
    for (int w = 1; w < nt; ++w) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    size_t nout = 0;
    for (size_t t = 0; t < nacc; ++t)
        for (const orc_candidate& c : per_trial[t]) {
            if (nout >= cap) return (size_t)-1;
            out[nout] = c;
            if (trial_of) trial_of[nout] = (int)t;
            ++nout;
        }
    if (seconds)
        *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return nout;
}

}  // extern "C"
