/*
 * orc_search.cpp -- candidate distillers and the per-DM search driver of
 * the FP64 CPU oracle.  TEST INFRASTRUCTURE ONLY (see psx_oracle.h).
 *
 * The distillers are written in C++ so that their S/N sort is the same
 * std::sort over the same comparator as the reference's
 * (include/transforms/distiller.hpp:16-48); std::sort is not stable, and
 * candidates with equal S/N must come out in the same order.
 */
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "psx_oracle.h"

namespace {

struct Cand {
    orc_candidate c;
    int tag;  /* position before sorting */
};

struct SnrGreater {
    bool operator()(const Cand& x, const Cand& y) const { return x.c.snr > y.c.snr; }
};

/* distiller.hpp:30-56: sort by descending S/N, then every candidate that
   is still unique removes the later candidates its condition matches.
   `cond(i, j)` returns the number of matches of j against survivor i (the
   reference appends one association per match when keep_related is set). */
template <class Cond>
size_t distill(orc_candidate* cands, size_t n, int* keep, int* nassoc, Cond cond)
{
    std::vector<Cand> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = Cand{cands[i], (int)i};
    std::sort(v.begin(), v.end(), SnrGreater());
    std::vector<char> uniq(n, 1);
    std::vector<int> na(n, 0);
    for (size_t i = 0; i < n; ++i) {
        if (!uniq[i]) continue;
        for (size_t j = i + 1; j < n; ++j) {
            int m = cond(v[i].c, v[j].c);
            if (m) { uniq[j] = 0; na[i] += m; }
        }
    }
    size_t kept = 0;
    for (size_t i = 0; i < n; ++i) {
        cands[i] = v[i].c;
        if (keep) keep[i] = uniq[i];
        if (nassoc) nassoc[i] = na[i];
        kept += uniq[i];
    }
    return kept;
}

}  // namespace

extern "C" {

/* distiller.hpp:63-108 (HarmonicDistiller::condition). */
size_t orc_harmonic_distill(orc_candidate* cands, size_t n, float tol,
                            float max_harm, int fractional_harms, int* keep,
                            int* nassoc)
{
    double upper = 1 + (double)tol, lower = 1 - (double)tol;
    return distill(cands, n, keep, nassoc,
                   [&](const orc_candidate& f, const orc_candidate& c) {
                       double fundi = f.freq, freq = c.freq;
                       float maxden = fractional_harms ? (float)std::pow(2.0, c.nh) : 1.0f;
                       int m = 0;
                       for (int jj = 1; (float)jj <= max_harm; ++jj)
                           for (int kk = 1; (float)kk <= maxden; ++kk) {
                               double ratio = kk * freq / (jj * fundi);
                               if (ratio > lower && ratio < upper) ++m;
                           }
                       return m;
                   });
}

/* distiller.hpp:115-163 (AccelerationDistiller::condition). */
size_t orc_accel_distill(orc_candidate* cands, size_t n, float tobs,
                         float tol, int* keep, int* nassoc)
{
    double tobs_over_c = (double)tobs / 299792458.0;
    return distill(cands, n, keep, nassoc,
                   [&](const orc_candidate& f, const orc_candidate& c) {
                       double fundi = f.freq, facc = f.acc;
                       double edge = fundi * tol;
                       double dacc = facc - c.acc;
                       float acc_freq = (float)(fundi + dacc * fundi * tobs_over_c);
                       if (acc_freq > fundi)
                           return (c.freq > fundi - edge && c.freq < acc_freq + edge) ? 1 : 0;
                       return (c.freq < fundi + edge && c.freq > acc_freq - edge) ? 1 : 0;
                   });
}

/* distiller.hpp:167-196 (DMDistiller::condition). */
size_t orc_dm_distill(orc_candidate* cands, size_t n, float tol, int* keep,
                      int* nassoc)
{
    double upper = 1 + (double)tol, lower = 1 - (double)tol;
    return distill(cands, n, keep, nassoc,
                   [&](const orc_candidate& f, const orc_candidate& c) {
                       double ratio = c.freq / (double)f.freq;
                       return (ratio > lower && ratio < upper) ? 1 : 0;
                   });
}

/* src/pipeline_multi.cu:161-290 for one DM trial, in FP64. */
size_t orc_search_dm(const float* series, size_t nsamps,
                     const orc_search_params* p, orc_candidate* out,
                     int* trial_of, size_t cap, orc_taps* taps)
{
    const size_t N = p->fft_size, B = N / 2 + 1;
    if (p->nharmonics < 0 || p->nharmonics > 5 || N < 16) return (size_t)-1;
    std::vector<double> tim(N, 0.0), tim_r(N), X(2 * B), pspec(B), med(B);
    size_t ncopy = std::min(nsamps, N);
    for (size_t i = 0; i < ncopy; ++i) tim[i] = series[i];
    orc_remove_baseline(tim.data(), ncopy);
    for (size_t i = ncopy; i < N; ++i) tim[i] = 0.0;

    /* pipeline_multi.cu:126-128: tobs and bin width are floats. */
    float tobs = (float)N * p->tsamp;
    float bwf = (float)(1.0 / (double)tobs);
    double bw = bwf;

    if (orc_rfft(tim.data(), N, X.data())) return (size_t)-1;
    orc_form_power(X.data(), B, pspec.data());
    orc_running_median(pspec.data(), B, bw, 0.05f, 0.5f, med.data());
    orc_deredden(X.data(), med.data(), B);
    if (p->nbirdies)
        orc_zap(X.data(), B, (float)bw, p->birdie_freqs, p->birdie_widths,
                p->nbirdies);
    orc_form_interbin(X.data(), B, pspec.data());
    double mean, rms, sd;
    orc_stats(pspec.data(), B, 0, &mean, &rms, &sd);
    if (orc_irfft(X.data(), N, tim.data())) return (size_t)-1;
    if (taps) {
        if (taps->tim_dered) std::memcpy(taps->tim_dered, tim.data(), sizeof(double) * N);
        if (taps->median) std::memcpy(taps->median, med.data(), sizeof(double) * B);
        taps->stats[0] = mean; taps->stats[1] = rms; taps->stats[2] = sd;
    }

    size_t nacc = orc_accel_list(p->acc_lo, p->acc_hi, p->acc_tol,
                                 p->acc_pulse_width, N, p->tsamp, p->cfreq,
                                 p->ch_bw, p->dm, p->cdm, nullptr, 0);
    std::vector<float> accs(nacc + 1);
    nacc = orc_accel_list(p->acc_lo, p->acc_hi, p->acc_tol, p->acc_pulse_width,
                          N, p->tsamp, p->cfreq, p->ch_bw, p->dm, p->cdm,
                          accs.data(), accs.size());

    const int F = p->nharmonics;
    std::vector<double> sums((size_t)F * B);
    std::vector<int> pidx(B);
    std::vector<double> psnr(B);
    std::vector<float> pfreq(B);
    double mean_n = mean * (double)N, sd_n = sd * (double)N;
    size_t nout = 0;
    for (size_t t = 0; t < nacc; ++t) {
        orc_resampleII(tim.data(), tim_r.data(), N, accs[t], p->tsamp,
                       p->resample_fused);
        if (orc_rfft(tim_r.data(), N, X.data())) return (size_t)-1;
        orc_form_interbin(X.data(), B, pspec.data());
        orc_normalise(pspec.data(), B, mean_n, sd_n);
        orc_harmonic_sums(pspec.data(), B, F, sums.data());
        if (taps && taps->tap_trial == (int)t) {
            if (taps->tim_r) std::memcpy(taps->tim_r, tim_r.data(), sizeof(double) * N);
            if (taps->pspec) std::memcpy(taps->pspec, pspec.data(), sizeof(double) * B);
            if (taps->sums) std::memcpy(taps->sums, sums.data(), sizeof(double) * F * B);
        }
        std::vector<orc_candidate> tc;
        for (int h = 0; h <= F; ++h) {
            const double* spec = h == 0 ? pspec.data() : sums.data() + (size_t)(h - 1) * B;
            size_t np = orc_find_peaks(spec, (unsigned)B, bw, h, p->min_snr,
                                       p->min_freq, p->max_freq, p->min_gap,
                                       pidx.data(), psnr.data(), pfreq.data(),
                                       B, nullptr);
            for (size_t k = 0; k < np; ++k)
                tc.push_back(orc_candidate{p->dm, p->dm_idx, accs[t], h,
                                           (float)psnr[k], pfreq[k]});
        }
        std::vector<int> keep(tc.size());
        orc_harmonic_distill(tc.data(), tc.size(), p->freq_tol, p->max_harm, 1,
                             keep.data(), nullptr);
        for (size_t k = 0; k < tc.size(); ++k) {
            if (!keep[k]) continue;
            if (nout >= cap) return (size_t)-1;
            out[nout] = tc[k];
            if (trial_of) trial_of[nout] = (int)t;
            ++nout;
        }
    }
    return nout;
}

}  // extern "C"
