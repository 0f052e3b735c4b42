// psx_host.cpp -- host-side logic of the search path: acceleration plan,
// peak ranges and clustering, candidate distillers.  No GPU involved.
//
// Compiled with -ffp-contract=off: the float arithmetic below decides
// which trials and bins exist and must round exactly as the reference's
// host code does.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "psx_host.h"

namespace psx {

// include/utils/utils.hpp:163-196 (dispersive smear, broadening, step),
// :198-232 (the list), every quantity in the reference's types.
std::vector<float> accel_list(float acc_lo, float acc_hi, float tol, float pulse_width,
                              size_t nsamps, float tsamp, float cfreq, float ch_bw, float dm,
                              float cdm)
{
    std::vector<float> out;
    ch_bw = std::fabs(ch_bw);
    if (acc_hi == acc_lo) {
        out.push_back(acc_hi);
        return out;
    }
    if (acc_hi >= 0 && acc_lo <= 0) out.push_back(0.0f);
    const float ftop = (float)((double)(cfreq + ch_bw / 2) / 1e9);
    const float fbot = (float)((double)(cfreq - ch_bw / 2) / 1e9);
    const float ddm = std::fabs(cdm - dm);
    const float inv = 1.0f / (fbot * fbot) - 1.0f / (ftop * ftop);
    const float tdm = (float)(4.15e-3 * (double)inv * (double)ddm);
    const float sumsq = (tdm * tdm) + (pulse_width * pulse_width) + (tsamp * tsamp);
    const float broad = (float)std::sqrt((double)sumsq);
    const float factor = (float)std::sqrt((double)(tol * tol) - 1.0);
    const float tobs = (float)nsamps * tsamp;
    const float step = (float)(2.0 * (double)broad * 24.0 * 299792458.0 /
                               (double)(tobs * tobs) * (double)factor);
    if (!(step > 0.0f)) return out;  // a zero step would never advance
    float acc = acc_lo;
    while (acc <= acc_hi) {
        out.push_back(acc);
        acc += step;
    }
    out.push_back(acc_hi);
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
    return out;
}

// include/transforms/peakfinder.hpp:78-91.
void peak_range(unsigned nbins, double bin_width, int nh, float min_freq, float max_freq,
                int* start, int* end, float* factor)
{
    const int size = (int)nbins;
    const float nyquist = (float)(bin_width * size);
    const int orig_size = (int)(2.0 * (size - 1.0));
    const double p2 = std::pow(2.0, nh);
    const int max_bin = (int)(((double)max_freq / bin_width) * p2);
    const int start_idx = (int)((double)((float)orig_size * (min_freq / nyquist)) * p2);
    *start = start_idx;
    *end = std::min(size, max_bin);
    *factor = (float)(1.0 / size * (double)nyquist / std::pow(2.0, (double)(float)nh));
}

// include/transforms/peakfinder.hpp:72-94: a cluster absorbs bins closer
// than min_gap to the bin holding its current maximum.
size_t unique_peaks(const int* idx, const float* snr, size_t count, int min_gap, int* oi,
                    float* os)
{
    size_t i = 0, np = 0;
    while (i < count) {
        float cpeak = snr[i];
        int cidx = idx[i], last = idx[i];
        ++i;
        while (i < count && (idx[i] - last) < min_gap) {
            if (snr[i] > cpeak) {
                cpeak = snr[i];
                cidx = idx[i];
                last = idx[i];
            }
            ++i;
        }
        oi[np] = cidx;
        os[np] = cpeak;
        ++np;
    }
    return np;
}

namespace {

struct SnrGreater {
    bool operator()(const psx_candidate& x, const psx_candidate& y) const { return x.snr > y.snr; }
};

// Number of (jj, kk) pairs with kk*freq/(jj*fundi) inside (lower, upper)
// for jj <= max_harm, kk <= maxden (distiller.hpp:75-84).  For each jj at
// most a couple of kk lie near jj*fundi/freq; only those are tested, with
// the reference's own expression, and a margin of one either side.
int harmonic_matches(double fundi, double freq, float max_harm, float maxden, double lower,
                     double upper, double tol)
{
    int m = 0;
    const bool fast = fundi > 0.0 && freq > 0.0 && std::isfinite(fundi) && std::isfinite(freq);
    for (int jj = 1; (float)jj <= max_harm; ++jj) {
        int k0 = 1, k1 = (int)maxden;
        if (fast) {
            const double x = jj * fundi / freq;
            const double lo = std::floor(x * (1.0 - 2.0 * tol)) - 1.0;
            const double hi = std::ceil(x * (1.0 + 2.0 * tol)) + 1.0;
            if (lo > k0) k0 = lo > 1e9 ? 1000000000 : (int)lo;
            if (hi < k1) k1 = hi < 0 ? 0 : (int)hi;
        }
        for (int kk = k0; kk <= k1 && (float)kk <= maxden; ++kk) {
            const double ratio = kk * freq / (jj * fundi);
            if (ratio > lower && ratio < upper) ++m;
        }
    }
    return m;
}

}  // namespace

// include/transforms/distiller.hpp:16-56 with the three conditions.
size_t distill(int kind, psx_candidate* c, size_t n, float tol, float max_harm, float tobs,
               int keep_related, int fractional, int* nassoc)
{
    std::sort(c, c + n, SnrGreater());
    std::vector<char> uniq(n, 1);
    std::vector<int> na(n, 0);
    // `1 + tolerance` with a float tolerance is a float sum in the reference
    // (distiller.hpp:76-77, 164-165), widened to double afterwards
    const double upper = (double)(1.0f + tol), lower = (double)(1.0f - tol);
    const double tobs_over_c = (double)tobs / 299792458.0;
    for (size_t i = 0; i < n; ++i) {
        if (!uniq[i]) continue;
        const double fundi = c[i].freq;
        for (size_t j = i + 1; j < n; ++j) {
            int m = 0;
            if (kind == PSX_DISTILL_HARMONIC) {
                const float maxden = fractional ? (float)std::pow(2.0, c[j].nh) : 1.0f;
                m = harmonic_matches(fundi, (double)c[j].freq, max_harm, maxden, lower, upper,
                                     (double)tol);
            } else if (kind == PSX_DISTILL_ACCEL) {
                const double edge = fundi * tol;
                const double dacc = (double)c[i].acc - c[j].acc;
                const double acc_freq = (float)(fundi + dacc * fundi * tobs_over_c);
                if (acc_freq > fundi)
                    m = (c[j].freq > fundi - edge && c[j].freq < acc_freq + edge) ? 1 : 0;
                else
                    m = (c[j].freq < fundi + edge && c[j].freq > acc_freq - edge) ? 1 : 0;
            } else {
                const double ratio = c[j].freq / fundi;
                m = (ratio > lower && ratio < upper) ? 1 : 0;
            }
            if (m) {
                uniq[j] = 0;
                na[i] += m;
            }
        }
    }
    size_t k = 0;
    for (size_t i = 0; i < n; ++i) {
        if (!uniq[i]) continue;
        c[k] = c[i];
        if (nassoc) nassoc[k] = keep_related ? na[i] : 0;
        ++k;
    }
    return k;
}

}  // namespace psx

extern "C" {

int psx_accel_list(float acc_lo, float acc_hi, float tol, float pulse_width_s, size_t nsamps,
                   float tsamp, float cfreq_hz, float ch_bw_hz, float dm, float cdm, float* h_out,
                   size_t cap, size_t* n)
{
    if (!n) return PSX_ERR_INVALID;
    std::vector<float> v = psx::accel_list(acc_lo, acc_hi, tol, pulse_width_s, nsamps, tsamp,
                                           cfreq_hz, ch_bw_hz, dm, cdm);
    *n = v.size();
    if (!h_out) return PSX_OK;
    if (v.size() > cap) return PSX_ERR_OVERFLOW;
    std::memcpy(h_out, v.data(), sizeof(float) * v.size());
    return PSX_OK;
}

int psx_peak_range(unsigned nbins, double bin_width, int nh, float min_freq, float max_freq,
                   int* start, int* end, float* factor)
{
    if (!start || !end || !factor) return PSX_ERR_INVALID;
    psx::peak_range(nbins, bin_width, nh, min_freq, max_freq, start, end, factor);
    return PSX_OK;
}

size_t psx_identify_unique_peaks(const int* idx, const float* snr, size_t count, int min_gap,
                                 int* out_idx, float* out_snr)
{
    if (!count) return 0;
    return psx::unique_peaks(idx, snr, count, min_gap, out_idx, out_snr);
}

size_t psx_distill(int kind, psx_candidate* cands, size_t n, float tol, float max_harm,
                   float tobs, int keep_related, int fractional, int* h_nassoc)
{
    if (!cands || !n) return 0;
    return psx::distill(kind, cands, n, tol, max_harm, tobs, keep_related, fractional, h_nassoc);
}

}  // extern "C"
