/*
 * psx_oracle.h -- FP64 CPU restatement of Peasoup's per-DM acceleration
 * search (the reference's src/kernels.cu stages, include/transforms/*.hpp
 * and the Worker loop of src/pipeline_multi.cu:111-303).
 *
 * TEST INFRASTRUCTURE ONLY.  The product never links, loads or calls this
 * code: it is the checker used by tests/, by the smoke test and by the
 * CPU-baseline leg of bench.py.
 *
 * Precision rule: sample and spectrum values are carried in double.  Every
 * quantity the reference computes on the host in float or in mixed
 * float/double arithmetic that steers control flow (acceleration list,
 * bin ranges, zap bins, median splice points, stretch weights, candidate
 * frequencies, resample index) is reproduced with exactly the reference's
 * types and operation order, so that those decisions match bit for bit.
 */
#ifndef PSX_ORACLE_H
#define PSX_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- transforms (orc_fft.c) ---- */
int orc_fft_c2c(double* data /* interleaved re,im */, size_t m, int sign);
int orc_rfft(const double* in, size_t n, double* out /* 2*(n/2+1) */);
int orc_irfft(const double* in /* 2*(n/2+1) */, size_t n, double* out);

/* ---- resampling (src/kernels.cu:315-386) ---- */
double orc_accel_fact(float acc, float tsamp);
void orc_resampleII_index(size_t n, float acc, float tsamp, int fused,
                          uint64_t* idx);
void orc_resampleII(const double* in, double* out, size_t n, float acc,
                    float tsamp, int fused);
void orc_resample_index(size_t n, float acc, float tsamp, int fused,
                        uint64_t* idx);

/* ---- spectrum forming (src/kernels.cu:216-259) ---- */
void orc_form_power(const double* X, size_t nbins, double* out);
void orc_form_interbin(const double* X, size_t nbins, double* out);

/* ---- dereddening (src/kernels.cu:902-1061, dereddener.hpp:41-66) ---- */
double orc_median3(double a, double b, double c);
double orc_median4(double a, double b, double c, double d);
double orc_median5(double a, double b, double c, double d, double e);
size_t orc_median_scrunch5(const double* in, size_t count, double* out);
void orc_linear_stretch(const double* in, size_t in_count, double* out,
                        size_t out_count);
void orc_splice_points(size_t nbins, double bin_width, float b5, float b25,
                       int* pos5, int* pos25);
void orc_running_median(const double* powers, size_t nbins, double bin_width,
                        float b5, float b25, double* median);
void orc_deredden(double* X, const double* median, size_t nbins);

/* ---- birdie zapping (birdiezapper.hpp:61-71, src/kernels.cu:1063-1096) */
void orc_zap_range(float freq, float width, float bin_width, unsigned nbins,
                   int* lo, int* hi);
void orc_zap(double* X, size_t nbins, float bin_width, const float* freqs,
             const float* widths, size_t nbirdies);

/* ---- statistics and normalisation (stats.hpp:6-43, kernels.cu:427-521) */
void orc_stats(const double* x, size_t n, size_t first, double* mean,
               double* rms, double* std);
void orc_normalise(double* x, size_t n, double mean, double sigma);
int orc_remove_baseline(double* x, size_t n);

/* ---- harmonic sums (src/kernels.cu:34-100) ---- */
int orc_harmonic_sums(const double* in, size_t n, int nfolds,
                      double* out /* nfolds*n */);

/* ---- peak finding (peakfinder.hpp:72-94) ---- */
void orc_peak_range(unsigned nbins, double bin_width, int nh, float min_freq,
                    float max_freq, int* start, int* end, float* factor);
size_t orc_identify_unique_peaks(const int* idx, const double* snr,
                                 size_t count, int min_gap, int* pidx,
                                 double* psnr);
size_t orc_find_peaks(const double* spec, unsigned nbins, double bin_width,
                      int nh, float thresh, float min_freq, float max_freq,
                      int min_gap, int* out_idx, double* out_snr,
                      float* out_freq, size_t cap, size_t* n_above);

/* ---- acceleration plan (include/utils/utils.hpp:143-233) ---- */
size_t orc_accel_list(float acc_lo, float acc_hi, float tol,
                      float pulse_width, size_t nsamps, float tsamp,
                      float cfreq, float ch_bw, float dm, float cdm,
                      float* out, size_t cap);

/* ---- candidates and distillers (candidates.hpp:10-17, distiller.hpp) -- */
typedef struct {
    float dm;
    int dm_idx;
    float acc;
    int nh;
    float snr;
    float freq;
} orc_candidate; /* same field order and size as the reference CandidatePOD */

/* Each distiller sorts `cands` in place by descending S/N (as the
   reference does before distilling) and writes keep[i] = 1 for the
   survivors, in the sorted order.  `assoc_parent` (may be NULL) receives,
   for every removed candidate, the index of the survivor that removed it
   (keep_related bookkeeping), else -1.  Returns the survivor count. */
size_t orc_harmonic_distill(orc_candidate* cands, size_t n, float tol,
                            float max_harm, int fractional_harms, int* keep,
                            int* assoc_parent);
size_t orc_accel_distill(orc_candidate* cands, size_t n, float tobs,
                         float tol, int* keep, int* assoc_parent);
size_t orc_dm_distill(orc_candidate* cands, size_t n, float tol, int* keep,
                      int* assoc_parent);

/* ---- the per-DM search (src/pipeline_multi.cu:161-294) ---- */
typedef struct {
    size_t fft_size;      /* N */
    float tsamp;          /* s */
    float dm, cdm;
    int dm_idx;
    float acc_lo, acc_hi, acc_tol, acc_pulse_width /* s */;
    float cfreq, ch_bw;   /* Hz */
    int nharmonics;       /* folds, 0..5 */
    float min_snr, min_freq, max_freq;
    int min_gap;
    float freq_tol, max_harm;
    const float* birdie_freqs;  /* may be NULL */
    const float* birdie_widths;
    size_t nbirdies;
    int resample_fused;   /* FMA contraction of the resample index */
} orc_search_params;

/* Per-trial debug taps: when tap_trial >= 0 the resampled series, the
   normalised interbinned spectrum and the harmonic sums of that trial are
   copied to the given buffers (any may be NULL). */
typedef struct {
    int tap_trial;
    double* tim_dered;   /* N   : dereddened series after C2R */
    double* tim_r;       /* N   : resampled series of the tapped trial */
    double* pspec;       /* B   : normalised interbinned spectrum */
    double* sums;        /* F*B : harmonic sums */
    double* median;      /* B   : running median of the prologue */
    double stats[3];     /* mean, rms, std of the prologue spectrum */
} orc_taps;

/* Runs one DM trial.  `cands` receives the per-trial harmonic-distilled
   candidates of every acceleration trial, in trial order (capacity cap).
   `trial_of` (may be NULL) receives the acceleration-trial index of each.
   Returns the number written, or (size_t)-1 on error / overflow. */
size_t orc_search_dm(const float* series, size_t nsamps,
                     const orc_search_params* p, orc_candidate* cands,
                     int* trial_of, size_t cap, orc_taps* taps);

#ifdef __cplusplus
}
#endif
#endif
