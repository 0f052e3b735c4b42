/*
 * peasoup_b200.h -- C ABI of the B200-native acceleration search.
 *
 * Drop-in boundary for Peasoup's per-DM acceleration-search path.  Each
 * entry point names the reference interface it replaces (file:line in
 * ewanbarr/peasoup).  Conventions, which differ from the reference on
 * purpose:
 *
 *   - Plain pointers and sizes only; "d_" arguments are device pointers,
 *     "h_" arguments host pointers.  Complex spectra are interleaved
 *     (re, im) float pairs, the layout of cufftComplex.
 *   - Every call returns an int status (PSX_OK == 0); psx_last_error()
 *     gives a message for the calling thread.  The reference threw
 *     std::runtime_error instead (include/utils/exceptions.hpp:64-74).
 *   - Device work is enqueued on the given CUDA stream (0 = legacy default
 *     stream) and is NOT followed by a device synchronisation; the
 *     reference synchronised after every launch.  Calls that return host
 *     values (psx_stats, psx_remove_baseline, psx_find_peaks,
 *     psx_search_dm) synchronise the given stream only.
 *   - Nothing here falls back to the CPU: without a usable CUDA device the
 *     calls fail with PSX_ERR_CUDA.
 */
#ifndef PEASOUP_B200_H
#define PEASOUP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* psx_stream_t; /* == cudaStream_t */

enum {
    PSX_OK = 0,
    PSX_ERR_INVALID = 1,     /* bad argument or size */
    PSX_ERR_CUDA = 2,        /* CUDA runtime error (incl. no device) */
    PSX_ERR_CUFFT = 3,       /* cuFFT error */
    PSX_ERR_ALLOC = 4,       /* device or host allocation failed */
    PSX_ERR_OVERFLOW = 5,    /* caller buffer too small; *n_out has the need */
    PSX_ERR_UNSUPPORTED = 6, /* valid request the library does not support */
    PSX_ERR_IO = 7,          /* file could not be read (zap list) */
    PSX_ERR_BUSY = 8         /* served loop: admission refused / queue full */
};

/* Message of the last failed call on this thread ("" if none). */
const char* psx_last_error(void);
/* Static text for a status code. */
const char* psx_status_string(int status);
/* Library version string. */
const char* psx_version(void);

/* ------------------------------------------------------------------ */
/* Stage kernels (one launch each, asynchronous on `stream`)           */
/* ------------------------------------------------------------------ */

/* out[i] = in[rn(i + i*k*(i-size))], k = float(acc*tsamp)/(2c) in double.
   Replaces device_resampleII (include/kernels/kernels.h:126, src/kernels.cu:355-369)
   behind TimeDomainResampler::resampleII (include/transforms/resampler.hpp:26-31). */
int psx_resampleII(const float* d_in, float* d_out, size_t size, float acc,
                   float tsamp, psx_stream_t stream);

/* Centred form: out[i] = in[rn(i + k*((i-size/2)^2 - (size/2)^2))].
   Replaces device_resample (kernels.h:118, src/kernels.cu:371-386) behind
   TimeDomainResampler::resample (resampler.hpp:19-24). */
int psx_resample(const float* d_in, float* d_out, size_t size, float acc,
                 float tsamp, psx_stream_t stream);

/* ntrials resampleII outputs of one input, d_out[t*size + i]; h_accs is a
   host array of ntrials accelerations.  Batched form of device_resampleII
   (no reference counterpart; the reference resamples one trial per call,
   src/pipeline_multi.cu:249). */
int psx_resampleII_batch(const float* d_in, float* d_out, size_t size,
                         const float* h_accs, int ntrials, float tsamp,
                         psx_stream_t stream);

/* way 0: amplitude |X_k| (z*rsqrtf(z), 0 where z == 0);
   way 1: interbinned amplitude sqrt(max(|X_k|^2, 0.5|X_k - X_{k-1}|^2)).
   Replaces device_form_power_series (kernels.h:111, src/kernels.cu:294-311)
   behind SpectrumFormer::form / form_interpolated (spectrumformer.hpp:8-22). */
int psx_form_power_series(const float* d_fseries, float* d_out, size_t nbins,
                          int way, psx_stream_t stream);

/* out[i] = median of in[5i..5i+4] for i < count/5; counts 1..4 give one
   value.  Replaces median_scrunch5 (kernels.h:252, src/kernels.cu:974-1008). */
int psx_median_scrunch5(const float* d_in, size_t count, float* d_out,
                        psx_stream_t stream);

/* Linear interpolation of in_count samples onto out_count.  Replaces
   linear_stretch (kernels.h:256, src/kernels.cu:1025-1038). */
int psx_linear_stretch(const float* d_in, size_t in_count, float* d_out,
                       size_t out_count, psx_stream_t stream);

/* Bytes of device scratch psx_running_median / psx_deredden need. */
size_t psx_running_median_scratch_bytes(size_t nbins);

/* Spliced 5/25/125-bin running median of an amplitude spectrum (splice at
   b5 and b25 Hz).  Replaces Dereddener::calculate_median
   (include/transforms/dereddener.hpp:41-62). */
int psx_running_median(const float* d_powers, size_t nbins, double bin_width,
                       float b5, float b25, float* d_median, void* d_scratch,
                       psx_stream_t stream);

/* X_k /= f_k (complex / real), bins 0..4 zeroed.  Replaces
   device_divide_c_by_f (kernels.h:262, src/kernels.cu:1040-1061) behind
   Dereddener::deredden (dereddener.hpp:64-66). */
int psx_divide_c_by_f(float* d_fseries, const float* d_f, size_t nbins,
                      psx_stream_t stream);

/* Running median of d_powers and the division of d_fseries by it in one
   pass (the median is never written).  Replaces the pair
   Dereddener::calculate_median + Dereddener::deredden
   (dereddener.hpp:41-66) as called at src/pipeline_multi.cu:213-217. */
int psx_deredden(float* d_fseries, const float* d_powers, size_t nbins,
                 double bin_width, float b5, float b25, void* d_scratch,
                 psx_stream_t stream);

/* Sets bins [floor((f-w)/bw), ceil((f+w)/bw)) of each birdie to 1+0i.
   Replaces device_zap_birdies (kernels.h:268, src/kernels.cu:1063-1096)
   behind Zapper::zap (birdiezapper.hpp:61-71). */
int psx_zap_birdies(float* d_fseries, const float* d_freqs,
                    const float* d_widths, float bin_width, size_t nbirdies,
                    size_t nbins, psx_stream_t stream);

/* Parses a zap list ("freq width" per line, birdiezapper.hpp:35-46) into
   host arrays.  With h_freqs == NULL only *n is set. */
int psx_read_zaplist(const char* path, float* h_freqs, float* h_widths,
                     size_t cap, size_t* n);

/* mean, rms and std = sqrt(rms^2 - mean^2) of d_x[first..n).  Synchronous
   (synchronises `stream`).  Replaces stats::stats / GPU_mean / GPU_rms
   (include/utils/stats.hpp:25-33, src/kernels.cu:433-461). */
int psx_stats(const float* d_x, size_t n, size_t first, float* h_mean,
              float* h_rms, float* h_std, psx_stream_t stream);

/* x = (x - mean) / sigma in place.  Replaces device_normalise
   (kernels.h:144, src/kernels.cu:496-521) behind stats::normalise
   (stats.hpp:35-40). */
int psx_normalise(float* d_x, float mean, float sigma, size_t n,
                  psx_stream_t stream);

/* Iterative mean removal (until |mean| <= 5e-7 n, at most 102 passes);
   synchronous.  Replaces GPU_remove_baseline (src/kernels.cu:463-479)
   behind DeviceTimeSeries::remove_baseline (timeseries.hpp:282-287).
   *h_passes (may be NULL) receives the number of passes. */
int psx_remove_baseline(float* d_x, size_t n, int* h_passes,
                        psx_stream_t stream);

/* d_x[0..n) = value.  Replaces GPU_fill (src/kernels.cu:482-488). */
int psx_fill(float* d_x, size_t n, float value, psx_stream_t stream);

/* Type conversion to float.  Replaces device_conversion<X,float>
   (kernels.h:322, src/kernels.cu:1171-1200). */
int psx_convert_u8_f32(const uint8_t* d_in, float* d_out, size_t n,
                       psx_stream_t stream);
int psx_convert_i8_f32(const int8_t* d_in, float* d_out, size_t n,
                       psx_stream_t stream);

/* Fractional harmonic sums: nharms (0..5) output spectra of n bins, output
   h_out_ptrs[h] = device pointer for fold h+1.  The pointer array is read
   on the host and passed by value (no copy to the device).  Replaces
   device_harmonic_sum (kernels.h:104, src/kernels.cu:34-100, 200-209)
   behind HarmonicFolder::fold (harmonicfolder.hpp:26-38). */
int psx_harmonic_sum(const float* d_in, float* const* h_out_ptrs, size_t n,
                     int nharms, psx_stream_t stream);

/* Order-preserving compaction of (index, value) pairs with value > thresh
   over [start, n) into device arrays of capacity `cap`; *h_count receives
   the number above threshold (may exceed cap: then PSX_ERR_OVERFLOW).
   Synchronous.  Replaces device_find_peaks (kernels.h:134-142,
   src/kernels.cu:398-423), whose Thrust types cannot cross a C ABI. */
int psx_find_peaks(const float* d_spec, int n, int start, float thresh,
                   int* d_idx, float* d_val, int cap, int* h_count,
                   psx_stream_t stream);

/* psx_find_peaks without any device allocation; no counterpart in the
   reference.  For callers that may not allocate GPU memory during a run
   (the device's memory is owned by their own pool or another framework,
   or allocation after start-up is forbidden so that memory use stays
   fixed).  Same arguments, results and errors as psx_find_peaks; the
   per-tile counts live in a 256 KiB array compiled into the library,
   which every GPU that loads the library holds until exit.  Limit:
   n - start <= 2^28 bins; larger requests fail with PSX_ERR_INVALID.
   The first call on each device looks up the array's device address with
   that device current and keeps it for the life of the process; make that
   first call before any stream capture.  A cudaDeviceReset invalidates
   the kept address: do not call this entry point in a process after a
   reset of the device.  All calls share the array: calls whose GPU work
   overlaps (different streams or host threads) race and give wrong
   results. */
int psx_find_peaks_noalloc(const float* d_spec, int n, int start, float thresh,
                           int* d_idx, float* d_val, int cap, int* h_count,
                           psx_stream_t stream);

/* Fused fractional harmonic sums, threshold test and compaction over `rows`
   normalised spectra of nbins bins (row r at d_spec + r*pitch; pitch a
   multiple of 4 floats, d_spec 16-byte aligned): for every fold h in
   0..nharms (0 = the spectrum itself) and bin i in [h_start[h], h_end[h])
   whose fold value exceeds `thresh`, one record of four ints {row, h, i,
   the value's float bits} is appended to d_records (order unspecified;
   the folds are never written).  Sums, scales and order are the
   reference's (src/kernels.cu:34-100); this replaces the pair
   HarmonicFolder::fold + PeakFinder's device_find_peaks per fold
   (harmonicfolder.hpp:26-38, kernels.cu:398-423).  *h_count = records (the
   need, with PSX_ERR_OVERFLOW).  Every barrier wait of the kernel is
   bounded by wait_limit polls (0 = the default); one that runs out makes
   the call fail with PSX_ERR_CUDA and a message, and leaves the context
   usable.  flags: 0, or 1 to stage nothing, so that the waits run out (a
   test of that path).  Synchronous. */
int psx_harmonic_peaks(const float* d_spec, size_t pitch, size_t nbins, int rows,
                       int nharms, const int* h_start, const int* h_end,
                       float thresh, int* d_records, size_t cap, size_t* h_count,
                       unsigned wait_limit, unsigned flags, psx_stream_t stream);

/* ------------------------------------------------------------------ */
/* Real transforms (cuFFT)                                             */
/* ------------------------------------------------------------------ */

typedef struct psx_fft_plan psx_fft_plan;
enum { PSX_FFT_R2C = 0, PSX_FFT_C2R = 1, PSX_FFT_C2C = 2 };

/* Unnormalised R2C / C2R plan of length `size`, `batch` transforms with
   input/output distances size and size/2+1, or (PSX_FFT_C2C) a complex
   plan of `batch` transforms of length `size`, distance size.  Replaces
   CuFFTerR2C / CuFFTerC2R (include/transforms/ffter.hpp:54-110) and
   CuFFTerC2C (ffter.hpp:33-53). */
int psx_fft_plan_create(psx_fft_plan** plan, size_t size, long long batch,
                        int kind);
/* Executes an R2C or C2R plan. */
int psx_fft_exec(psx_fft_plan* plan, const void* d_in, void* d_out,
                 psx_stream_t stream);
/* Executes a PSX_FFT_C2C plan in `direction` -1 (forward, CUFFT_FORWARD)
   or +1 (inverse, CUFFT_INVERSE), unnormalised; in place when d_in ==
   d_out.  Replaces CuFFTerC2C::execute (ffter.hpp:43-47). */
int psx_fft_exec_c2c(psx_fft_plan* plan, const void* d_in, void* d_out, int direction,
                     psx_stream_t stream);
int psx_fft_plan_destroy(psx_fft_plan* plan);

/* ------------------------------------------------------------------ */
/* Host logic (no GPU)                                                 */
/* ------------------------------------------------------------------ */

/* Same field order and size as the reference's CandidatePOD
   (include/data_types/candidates.hpp:10-17), the record written to
   candidates.peasoup. */
typedef struct {
    float dm;
    int dm_idx;
    float acc;
    int nh;
    float snr;
    float freq;
} psx_candidate;

/* Acceleration trial list of one DM.  Replaces
   AccelerationPlan::generate_accel_list (include/utils/utils.hpp:198-232);
   all arithmetic in float as there.  With h_out == NULL only *n is set. */
int psx_accel_list(float acc_lo, float acc_hi, float tol, float pulse_width_s,
                   size_t nsamps, float tsamp, float cfreq_hz, float ch_bw_hz,
                   float dm, float cdm, float* h_out, size_t cap, size_t* n);

/* Search range [*start, *end) and frequency factor of a spectrum with
   harmonic number nh.  Restates peakfinder.hpp:78-91. */
int psx_peak_range(unsigned nbins, double bin_width, int nh, float min_freq,
                   float max_freq, int* start, int* end, float* factor);

/* Cluster sorted above-threshold bins (min_gap rule of
   PeakFinder::identify_unique_peaks, peakfinder.hpp:72-94). */
size_t psx_identify_unique_peaks(const int* idx, const float* snr,
                                 size_t count, int min_gap, int* out_idx,
                                 float* out_snr);

enum { PSX_DISTILL_HARMONIC = 0, PSX_DISTILL_ACCEL = 1, PSX_DISTILL_DM = 2 };

/* Candidate distillation in place: cands are sorted by descending S/N and
   the survivors are moved to the front, in that order; returns their
   count.  h_nassoc (may be NULL, n entries) receives each survivor's
   association count (Candidate::count_assoc when keep_related is set).
   kind HARMONIC: HarmonicDistiller(tol, max_harm, keep_related,
   fractional) (distiller.hpp:63-108); ACCEL: AccelerationDistiller(tobs,
   tol, keep_related) (:115-163); DM: DMDistiller(tol, keep_related)
   (:167-196). */
size_t psx_distill(int kind, psx_candidate* cands, size_t n, float tol,
                   float max_harm, float tobs, int keep_related,
                   int fractional, int* h_nassoc);

/* ------------------------------------------------------------------ */
/* Candidate forests: the association trees of the distillers           */
/* ------------------------------------------------------------------ */

/* A candidate forest is `nodes` in depth-first order with sizes[i] = the
   number of nodes in the subtree node i roots (itself included); roots are
   the nodes that start a top-level subtree.  It is the reference's
   Candidate::assoc tree (include/data_types/candidates.hpp:19-86) laid out
   as Candidate::collect_candidates walks it, so a root's subtree is the
   run of records candidates.peasoup holds for that candidate, and
   sizes[root] - 1 is its Candidate::count_assoc(). */

/* Distillation of the roots of a forest, keeping trees: BaseDistiller::
   distill (include/transforms/distiller.hpp:25-57) with the three
   conditions as in psx_distill; with keep_related each survivor's subtree
   is its own followed by every absorbed candidate's (in the reference's
   append order, repeated where it appends more than once).  Survivors come
   out in descending S/N.  *n_out = nodes written (the need, with
   PSX_ERR_OVERFLOW), *n_roots = survivors (may be NULL).  Replaces the
   global DMDistiller / HarmonicDistiller(keep_related) of
   src/pipeline_multi.cu:406-407, 547-548. */
int psx_distill_forest(int kind, const psx_candidate* nodes, const int* sizes,
                       size_t n_nodes, float tol, float max_harm, float tobs,
                       int keep_related, int fractional, psx_candidate* h_out,
                       int* h_out_sizes, size_t cap, size_t* n_out,
                       size_t* n_roots);

typedef struct {
    int is_physical;       /* 1/freq > channel DM smearing at the DM */
    int is_adjacent;       /* an association one DM trial away, or none off-DM */
    float ddm_count_ratio; /* share of associations within the DM width */
    float ddm_snr_ratio;   /* share of their S/N */
    int nassoc;            /* Candidate::count_assoc() */
} psx_candidate_score;

/* CandidateScorer(tsamp, cfreq, foff, bw)::score for every root, from its
   direct associations (include/transforms/scorer.hpp:8-87; frequencies in
   MHz as the reference passes them, src/pipeline_multi.cu:550-552). */
int psx_score_forest(const psx_candidate* nodes, const int* sizes,
                     size_t n_nodes, float tsamp, float cfreq, float foff,
                     float bw, psx_candidate_score* h_scores, size_t cap,
                     size_t* n_roots);

/* candidates.peasoup: per root an int record count and its subtree's
   24-byte records (CandidateFileWriter::write_binary, include/utils/
   output_stats.hpp:270-298; no FOLD blocks: folding is not part of this
   library).  h_offsets (may be NULL) receives each root's byte offset. */
int psx_write_candidates(const char* path, const psx_candidate* nodes,
                         const int* sizes, size_t n_nodes, long long* h_offsets,
                         size_t cap, size_t* n_roots);

/* overview.xml (OutputFileWriter, include/utils/output_stats.hpp:20-210),
   built section by section and written in the reference's XML layout
   (include/utils/xml_util.hpp).  Sections whose values come from outside
   this library (header_parameters, search_parameters,
   segment_parameters, execution_times) are added as name/value pairs,
   values already formatted. */
typedef struct psx_overview psx_overview;
int psx_overview_create(psx_overview** out);
void psx_overview_destroy(psx_overview* o);
int psx_overview_add_section(psx_overview* o, const char* section,
                             const char* const* keys, const char* const* values,
                             size_t n);
int psx_overview_add_misc_info(psx_overview* o, long long unix_time);
int psx_overview_add_dm_list(psx_overview* o, const float* dms, size_t n);
int psx_overview_add_acc_list(psx_overview* o, const float* accs, size_t n,
                              float cdm);
int psx_overview_add_device_info(psx_overview* o, int runtime_version,
                                 int driver_version, const int* ids,
                                 const char* const* names, const int* major,
                                 const int* minor, size_t n);
int psx_overview_add_candidates(psx_overview* o, const psx_candidate* nodes,
                                const int* sizes, size_t n_nodes,
                                const psx_candidate_score* scores,
                                const long long* byte_offsets);
/* Writes the document to `path` (may be NULL) and/or copies it into h_text
   (cap bytes, NUL-terminated; may be NULL); *n_text = its length. */
int psx_overview_write(psx_overview* o, const char* path, char* h_text,
                       size_t cap, size_t* n_text);

/* ------------------------------------------------------------------ */
/* Per-DM acceleration search (the fused hot path)                     */
/* ------------------------------------------------------------------ */

enum {
    PSX_MODE_PLAIN = 0,   /* one acceleration trial per launch sequence */
    PSX_MODE_BATCHED = 1  /* many trials per launch, graph-captured */
};

typedef struct {
    size_t fft_size;           /* N: 2^k or 3*2^k, 1024 <= N <= 2^28 */
    float tsamp;               /* s */
    float cdm;                 /* coherent DM of the acceleration plan */
    float acc_lo, acc_hi;      /* m/s^2 */
    float acc_tol;             /* AccelerationPlan tolerance (1.10) */
    float acc_pulse_width;     /* s (64e-6) */
    float cfreq_hz, ch_bw_hz;  /* centre frequency and channel width */
    int nharmonics;            /* folds, 0..5 (4) */
    float min_snr;             /* (9) */
    float min_freq, max_freq;  /* Hz (0.1, 1100) */
    int min_gap;               /* bins (30) */
    float freq_tol;            /* (1e-4) */
    float max_harm;            /* (16) */
    float boundary_5_freq;     /* (0.05) */
    float boundary_25_freq;    /* (0.5) */
    const float* birdie_freqs; /* host, may be NULL */
    const float* birdie_widths;
    size_t nbirdies;
    int mode;                  /* PSX_MODE_* */
    int batch;                 /* trials per launch (batched; rounded down to a
                                  power of two unless the two-pass transform
                                  carries the trials); 0 = default */
    int use_fft_callback;      /* must be 0: the resample inside cuFFT needs LTO
                                  load callbacks, which cuFFT 11.4 (CUDA 12.9)
                                  cannot plan on sm_100; a non-zero value is
                                  refused with PSX_ERR_UNSUPPORTED.  The
                                  two-pass transform (fft_form 3) does that
                                  fusion itself */
    int use_graph;             /* batched: capture the trial schedule */
    int harm_shape;            /* harmonic-kernel tile shape 1..PSX_HARM_SHAPES;
                                  0 = default (psx_autotune picks one) */
    int lanes;                 /* batched: launch groups alternate over this
                                  many streams with their own buffers, so one
                                  group's harmonic sums overlap the next one's
                                  transform (1 or 2; 0 = 1) */
    int fft_form;              /* batched: 0 = default (3 where fft_size allows
                                  it, else 1); 1 = cuFFT complex transform of
                                  the series read as interleaved pairs, then
                                  one kernel that unpacks the real spectrum,
                                  interbins and normalises; 2 = the reference's
                                  real transform, then interbin + normalise;
                                  3 = the library's own two-pass transform of
                                  the interleaved pairs with the resample
                                  gather in its first pass, then the unpack
                                  kernel (fft_size 2^19 .. 2^25 or
                                  3 * 2^17 .. 3 * 2^23) */
    int group_dms;             /* batched: DM trials of a psx_search_block
                                  call whose per-DM prologues (baseline
                                  removal through the inverse transform) run
                                  as one batch of row-indexed launches and
                                  batched cuFFT plans (with fft_form 3 their
                                  acceleration trials then run as one list,
                                  in launch groups across the DM trials).
                                  0 = default: 4 when
                                  fft_size <= 2^22 and the call's DM trials
                                  average at most 32 acceleration trials,
                                  else off; 1 = off; 2..16 = that many
                                  whenever the call has more DM trials than
                                  that.  Results do not depend on it. */
} psx_search_config;

/* Number of tile shapes of the fused harmonic-sum kernel (tile bins,
   consumer threads, CTAs per SM, exact pass in or out of line; shapes 6
   and 7 stage each tile for 3 or 2 trials at once with 2D tensor copies
   and need the batched mode with at least that many trials per group). */
#define PSX_HARM_SHAPES 7

/* Fills `cfg` with the reference's defaults (include/utils/cmdline.hpp:
   99-191) for a transform of `fft_size` samples of `tsamp` s. */
void psx_search_config_defaults(psx_search_config* cfg, size_t fft_size,
                                float tsamp);

typedef struct psx_search psx_search;

/* Device memory one search instance holds (admission model). */
size_t psx_search_footprint(const psx_search_config* cfg);

/* Allocates buffers and plans for `cfg` on the current device.  Replaces
   the per-thread set-up of Worker::start (src/pipeline_multi.cu:114-152). */
int psx_search_create(const psx_search_config* cfg, psx_search** s);
int psx_search_destroy(psx_search* s);
/* Stream used by the instance (default: a private non-blocking stream). */
int psx_search_set_stream(psx_search* s, psx_stream_t stream);

enum {
    PSX_OUT_TRIAL = 0,  /* per-trial harmonic-distilled candidates */
    PSX_OUT_DM = 1,     /* plus the per-DM acceleration distillation:
                           the reference Worker's dm_trial_cands */
    PSX_OUT_DM_FOREST = 2 /* the same survivors with their association
                             trees: a candidate forest (see psx_distill_forest)
                             whose subtree sizes go to h_nassoc */
};

/* Searches one dedispersed series: the body of the reference's DM loop,
   src/pipeline_multi.cu:161-294 (copy, baseline removal, padding, R2C,
   dereddening, zapping, statistics, C2R, then every acceleration trial:
   resample, R2C, interbinning, normalisation, harmonic sums, peak
   finding, harmonic distillation).  `series` is host memory unless
   series_on_device.  Candidates are written to h_out in the reference's
   order; h_nassoc (may be NULL) gets association counts (PSX_OUT_DM);
   h_trial (may be NULL) gets each candidate's acceleration-trial index.
   Synchronous.  PSX_ERR_OVERFLOW when cap is too small (*n_out = need). */
int psx_search_dm(psx_search* s, const float* series, size_t nsamps,
                  int series_on_device, float dm, int dm_idx, int output,
                  psx_candidate* h_out, int* h_nassoc, int* h_trial,
                  size_t cap, size_t* n_out);

/* Searches `ndm` dedispersed series (series[d], host pointers unless
   series_on_device) of the same length: the reference Worker's DM loop
   (src/pipeline_multi.cu:155-295) for a block of DM trials.  The host
   clusters and distils DM d while the GPU already searches DM d+1.
   Output as psx_search_dm for every DM in turn; h_dm (may be NULL)
   receives each candidate's position in the block.  Synchronous. */
int psx_search_block(psx_search* s, const float* const* series, size_t nsamps,
                     int series_on_device, const float* dms, const int* dm_idx,
                     int ndm, int output, psx_candidate* h_out, int* h_nassoc,
                     int* h_trial, int* h_dm, size_t cap, size_t* n_out);

/* Autotuner; no counterpart in the reference (which has one fixed
   schedule).  Times the batched search of `cfg` on seeded synthetic noise
   of cfg->fft_size samples for every pair (trials per launch group from
   h_batches[0..nbatch), harmonic-kernel shape 1..PSX_HARM_SHAPES): one
   warm-up DM trial, then `reps` DM trials through psx_search_block, timed
   on the host.  When the DM-0 acceleration list is longer than max_trials
   the range is narrowed around its middle for the timing.  Candidates whose
   footprint exceeds 80 % of the free device memory are skipped.  Writes
   the fastest pair into cfg->batch and cfg->harm_shape; h_ms (may be NULL)
   receives nbatch * PSX_HARM_SHAPES milliseconds per DM trial, batch-major
   (-1 for a skipped pair: one that does not fit, or that the configuration
   cannot use, e.g. a multi-trial harmonic shape with fewer trials per
   group).  Results never depend on the pair chosen. */
int psx_autotune(psx_search_config* cfg, const int* h_batches, int nbatch,
                 int reps, int max_trials, double* h_ms);

typedef struct {
    int ntrials;          /* acceleration trials of the last call */
    int nbatches;         /* launch groups of the last call */
    int kernel_launches;  /* kernels this library launched */
    int fft_launches;     /* cuFFT executions */
    long long above_threshold; /* (bin, fold) pairs above threshold */
    int fft_callback;     /* always 0 (see use_fft_callback) */
    int graph;            /* 1 if the trial schedule ran as a CUDA graph */
    int batch;            /* trials per launch used */
    int baseline_passes;  /* mean-removal passes of the last DM (-1: host loop) */
    int harm_shape;       /* harmonic-kernel tile shape in use */
    int capture_fallbacks; /* schedules launched directly because their
                              graph capture was invalidated */
    int fft_form;         /* transform path of the trials: 1 cuFFT complex
                             transform + fused unpack, 2 real transform (the
                             reference's), 3 the library's own two-pass
                             transform with the resample in its first pass */
    int group_dms;        /* DM trials per grouped prologue in the last call
                             (0: one prologue per DM trial) */
} psx_search_info;

int psx_search_last_info(const psx_search* s, psx_search_info* info);

/* Per-stage device time from CUDA events recorded on the instance's
   stream around every launch group (when enabled). */
typedef struct {
    double prologue_ms;   /* per-DM prologue */
    double resample_ms;   /* resample gathers (fft_form 3: the first pass of
                             the two-pass transform, which does the gather) */
    double fft_ms;        /* trial transforms (fft_form 3: the second pass) */
    double form_ms;       /* interbin + normalise */
    double harm_ms;       /* harmonic sums + threshold + compaction */
    long long groups;     /* launch groups timed */
    long long trials;     /* acceleration trials timed */
    long long dms;        /* DM trials timed */
    long long event_errors; /* event pairs that could not be timed */
    int last_event_error;   /* cudaError_t of the last such pair */
    /* host time of the calling thread (wall clock, recorded always):
       queuing each DM trial's work, blocked waiting for a DM trial's device
       work to finish, and reading back + distilling its records */
    double host_enqueue_ms;
    double host_wait_ms;
    double host_collect_ms;
} psx_search_profile;

/* Scheduling hint for a server running several instances on one device
   (no counterpart in the reference, which runs one search per GPU): with
   `high` set, the instance's kernels go to streams of the device's greatest
   priority, so that, where two searches share the GPU, its CTAs are
   scheduled first.  Takes effect at the next DM trial the instance starts;
   applies to instances on their own streams (not after
   psx_search_set_stream).  Safe to call from another thread while a search
   runs. */
int psx_search_set_priority(psx_search* s, int high);

int psx_search_set_profile(psx_search* s, int on);
int psx_search_get_profile(psx_search* s, psx_search_profile* out, int reset);

/* Debug tap: the dereddened series of the last call (N floats, scaled by
   N as the reference leaves it) and, for trial `trial` of the last call,
   its resampled series (N floats) and normalised interbinned spectrum
   (N/2+1 floats), recomputed on the device through the instance's own
   transform path (psx_search_info::fft_form; with the two-pass transform
   the series is what its first pass gathers, dumped instead of
   transformed).  Any pointer may be NULL. */
int psx_search_debug_tap(psx_search* s, int trial, float* h_tim_dered,
                         float* h_tim_r, float* h_pspec, float* h_norm2);

/* Reuses an instance for another request with the same transform length,
   mode, batch, harmonic shape, lanes, transform path and prologue
   grouping rows (the things its buffers and plans depend on): fold count,
   acceleration range, tsamp, thresholds,
   frequency limits and birdies may all change.  Waits for the instance's
   queued work first.  No counterpart in the reference (whose Worker builds
   its transforms once per process, src/pipeline_multi.cu:114-149). */
int psx_search_retarget(psx_search* s, const psx_search_config* cfg);

/* ------------------------------------------------------------------ */
/* Served loop; no counterpart in the reference, which searches one     */
/* observation per process                                              */
/* ------------------------------------------------------------------ */

typedef struct psx_server psx_server;

typedef struct {
    int device;         /* CUDA device of every search instance */
    size_t hbm_budget;  /* device bytes the server may hold in instances
                           (busy and pooled), by psx_search_footprint */
    int max_active;     /* requests searched at once (1..64), one host thread
                           and one instance each; their GPU work overlaps */
    int max_queue;      /* pending requests before submit refuses */
    int policy;         /* scheduling between running requests:
                           PSX_SERVE_LEAST_WORK (0) -- the one with the least
                           work at the device's greatest stream priority;
                           PSX_SERVE_EVEN (1) -- no priority hint: running
                           requests share the device evenly;
                           PSX_SERVE_EXCLUSIVE (2) -- one request on the
                           device at a time (more worker threads only wait),
                           admitted least work first, a request passed
                           over 8 times next; measured best on mixed
                           request streams (the Python Server's default) */
} psx_server_config;

enum { PSX_SERVE_LEAST_WORK = 0, PSX_SERVE_EVEN = 1, PSX_SERVE_EXCLUSIVE = 2 };

typedef struct {
    double t_submit;    /* seconds on the server clock (psx_server_clock) */
    double t_admit;     /* when a slot and the memory were granted */
    double t_done;      /* when its candidates were ready */
    size_t footprint;   /* bytes newly charged at admission (0 if reused) */
    long long ntrials;  /* acceleration trials searched */
    int ndm;            /* DM trials */
    int status;         /* PSX_OK or the failure */
    int engine_reused;  /* 1 if a pooled instance was retargeted */
} psx_request_stats;

/* Starts max_active worker threads on `device`. */
int psx_server_create(const psx_server_config* cfg, psx_server** out);
/* Fails requests not yet admitted (PSX_ERR_BUSY), lets admitted ones
   finish, and frees every instance. */
int psx_server_destroy(psx_server* srv);
/* Seconds since the server was created. */
double psx_server_clock(psx_server* srv);

/* Queues a search of ndm DM trials: series[d] holds nsamps floats (device
   or host memory per series_on_device) and must stay valid until the
   request completes; the config (birdies included) is copied.  Requests
   are admitted first in, first out, when a worker is free and the new
   instance they need fits the budget (a pooled instance with the same
   shape is reused).  With policy PSX_SERVE_LEAST_WORK, of the requests
   running at once the one with the least work (acceleration trials times
   transform length over its DM trials) runs at the higher stream priority
   (psx_search_set_priority); with PSX_SERVE_EVEN they share the device
   without a hint.  With PSX_SERVE_EXCLUSIVE one request runs at a time,
   to completion; the next is the pending one with the least work, unless
   one has been passed over 8 times (the oldest of those then goes first).
   PSX_ERR_BUSY: queue full; PSX_ERR_ALLOC: larger than the whole budget. */
int psx_server_submit(psx_server* srv, const psx_search_config* cfg,
                      const float* const* series, size_t nsamps,
                      int series_on_device, const float* dms,
                      const int* dm_idx, int ndm, long long* ticket);

/* Waits up to timeout_s seconds (< 0: no limit) for a request and copies
   its per-DM acceleration-distilled candidates in DM order (the output of
   psx_search_block with PSX_OUT_DM), their association counts and DM
   positions (h_nassoc, h_dm and stats may be NULL).  PSX_ERR_BUSY: still
   running; PSX_ERR_OVERFLOW: *n_out is the need, call again.  The ticket
   is released once its result (or failure) has been returned. */
int psx_server_wait(psx_server* srv, long long ticket, double timeout_s,
                    psx_candidate* h_out, int* h_nassoc, int* h_dm,
                    size_t cap, size_t* n_out, psx_request_stats* stats);

/* Bytes held, requests running, waiting, and pooled idle instances. */
int psx_server_status(psx_server* srv, size_t* used_bytes, int* active,
                      int* pending, int* pooled);

/* ------------------------------------------------------------------ */
/* Producer side: SIGPROC filterbank input and dedispersion            */
/* ------------------------------------------------------------------ */

/* The keywords of a SIGPROC header (SigprocHeader,
   include/data_types/header.hpp:171-212); unset values are zero. */
typedef struct {
    char source_name[80];
    char rawdatafile[80];
    double az_start, za_start, src_raj, src_dej, tstart, tsamp, period;
    double fch1, foff, refdm;
    int nchans, telescope_id, machine_id, data_type, ibeam, nbeams, nbits;
    int barycentric, pulsarcentric, nbins, nsamples, nifs, npuls;
    unsigned char signed_data;
    size_t header_size; /* bytes before the first sample */
} psx_sigproc_header;

/* Reads the header of a SIGPROC file.  nsamples == 0 in the file is
   replaced by (file size - header size) / nchans * 8 / nbits.  Unknown
   keywords are skipped with a warning on stderr, as the reference does.
   Replaces read_header (include/data_types/header.hpp:339-403) behind the
   SigprocFilterbank constructor (include/data_types/filterbank.hpp:261-300).
   PSX_ERR_IO: unreadable file or no HEADER_START. */
int psx_sigproc_read_header(const char* path, psx_sigproc_header* h);

/* Parses a SIGPROC header held in memory (the first n bytes of a file);
   nsamples is left as the header gives it.  PSX_ERR_OVERFLOW: the bytes
   end before HEADER_END (read more and call again); PSX_ERR_IO: not a
   SIGPROC header.  The parsing half of read_header
   (include/data_types/header.hpp:339-392). */
int psx_sigproc_parse_header(const void* h_bytes, size_t n, psx_sigproc_header* h);

/* Reads up to nsamples sample rows starting at start_sample into h_dst
   (nsamples * nchans * nbits / 8 bytes); *h_nread = rows read (fewer at
   the end of the file).  Replaces SigprocFilterbank::load_gulp
   (include/data_types/filterbank.hpp:308-328). */
int psx_sigproc_read(const char* path, const psx_sigproc_header* h, size_t start_sample,
                     size_t nsamples, void* h_dst, size_t* h_nread);

/* Writes a SIGPROC header (HEADER_START, the set keywords, HEADER_END)
   to a new file and returns its size in *h_size.  The writer side of
   header_write (include/data_types/header.hpp:222-300). */
int psx_sigproc_write_header(const char* path, const psx_sigproc_header* h,
                             size_t* h_size);

/* Reads a DM list, one value per line; an empty line repeats the previous
   value (0 for a leading empty line), as getFileContent does
   (src/pipeline_multi.cu:313-337).  PSX_ERR_OVERFLOW: *n_out = need. */
int psx_read_dm_file(const char* path, float* h_out, size_t cap, size_t* n_out);

/* Direct incoherent dedispersion plan (dedisp_plan behind Dedisperser,
   include/transforms/dedisperser.hpp:13-188).  The plan owns its device
   scratch (channel-major samples, shift tables), grown on first use. */
typedef struct psx_dedisp_plan psx_dedisp_plan;

/* dedisp_create_plan_multi(nchans, tsamp, fch1, foff): per-channel delays
   of 4.15e3/tsamp * (f_c^-2 - fch1^-2) samples per unit DM, f_c = fch1 +
   c*foff (MHz).  foff must be negative (fch1 the highest frequency). */
int psx_dedisp_create(size_t nchans, float tsamp, float fch1, float foff,
                      psx_dedisp_plan** out);
int psx_dedisp_destroy(psx_dedisp_plan* plan);
/* Dedisperser::set_dm_list (dedisperser.hpp:43-57). */
int psx_dedisp_set_dm_list(psx_dedisp_plan* plan, const float* h_dms, size_t n);
/* Dedisperser::generate_dm_list (dedisperser.hpp:63-71): DMs from dm_start
   upward, each step the largest whose smearing, combined with the pulse
   width (microseconds) and sampling time, stays within `tol` times the
   width at the previous DM; the last DM is the first at or past dm_end. */
int psx_dedisp_generate_dm_list(psx_dedisp_plan* plan, float dm_start, float dm_end,
                                float width_us, float tol);
size_t psx_dedisp_get_dm_count(const psx_dedisp_plan* plan);
int psx_dedisp_get_dm_list(const psx_dedisp_plan* plan, float* h_out, size_t cap);
int psx_dedisp_get_delay_table(const psx_dedisp_plan* plan, float* h_out);
/* Dedisperser::set_killmask (dedisperser.hpp:73-110): h_mask[c] == 0 drops
   channel c from every sum; NULL restores all channels. */
int psx_dedisp_set_killmask(psx_dedisp_plan* plan, const int* h_mask);
/* Samples the largest DM delays the last channel by (rounded half up);
   each output series is nsamps - max_delay long. */
size_t psx_dedisp_get_max_delay(const psx_dedisp_plan* plan);

/* Upper bound on the plan's channel-major scratch (default 4 GiB): longer
   inputs are dedispersed in time gulps that overlap by the maximum delay,
   as Dedisperser::dedisperse gulps (dedisperser.hpp:112-186). */
int psx_dedisp_set_scratch_limit(psx_dedisp_plan* plan, size_t bytes);

#define PSX_DEDISP_RAW 1 /* output the plain channel sums */

/* Dedisperses nsamps SIGPROC sample rows (device memory, nchans*nbits/8
   bytes each; nbits 1, 2, 4, 8 or 16) into d_out: row d (DM trial d of the
   list), out_pitch floats apart, holds nsamps - max_delay samples.  The
   channel sums are exact integers; unless PSX_DEDISP_RAW they are mapped
   to (sum - nchans*m/2) / (m*sqrt(nchans)) + 1/2, m = 2^nbits - 1.
   d_out must be 16-byte aligned and out_pitch a multiple of 4.
   Asynchronous on `stream`.  Replaces dedisp_execute
   (dedisperser.hpp:148-156) with the block left in device memory for the
   search, where the reference copied it to the host. */
int psx_dedisp_execute(psx_dedisp_plan* plan, size_t nsamps, const uint8_t* d_in,
                       int nbits, float* d_out, size_t out_pitch, int flags,
                       psx_stream_t stream);

/* As psx_dedisp_execute with the sample rows in host memory: the rows
   cross to the device in pieces that overlap the unpacking of the
   previous piece.  Pinned h_in gives asynchronous copies. */
int psx_dedisp_execute_host(psx_dedisp_plan* plan, size_t nsamps, const uint8_t* h_in,
                            int nbits, float* d_out, size_t out_pitch, int flags,
                            psx_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* PEASOUP_B200_H */
