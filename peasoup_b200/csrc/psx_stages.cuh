// psx_stages.cuh -- launchers of the single-stage kernels, shared with the
// search engine (psx_search.cu).  All are asynchronous on `s`.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace psx {

double accel_fact(float acc, float tsamp);

// ntrials outputs; trial t uses d_ktab[t] (or k when d_ktab is null) and is
// written at d_out + t*out_pitch.
int launch_resample(const float* d_in, float* d_out, size_t n, const double* d_ktab, double k,
                    int ntrials, size_t out_pitch, bool centred, cudaStream_t s);

size_t median_scratch_bytes(size_t nbins);

// Median levels + splice; writes the median (d_median) and/or divides the
// spectrum d_X by it (bins 0..4 zeroed).
int launch_running_median(const float* d_powers, size_t nbins, double bin_width, float b5,
                          float b25, float* d_median, float* d_X, void* d_scratch,
                          cudaStream_t s);

int launch_zap(float* d_X, const float* d_freqs, const float* d_widths, float bin_width,
               size_t nbirdies, size_t nbins, cudaStream_t s);

int reduction_blocks();

// Sums of x (or of the interbinned amplitude of the complex spectrum x)
// over [first, n); d_stat (5 floats) receives mean, rms, std,
// mean*scale, std*scale.
int launch_stats(const float* d_x, bool interbinned, size_t first, size_t n, double2* d_partials,
                 double* d_sums, float* d_stat, float scale, cudaStream_t s);

int remove_baseline_pass(float* d_x, size_t n, double2* d_partials, double* d_sums,
                         float* d_mean, cudaStream_t s);

int launch_fill(float* d_x, size_t n, float value, cudaStream_t s);

// Per-block partial sums of x and x^2 over [0, n) (reduction_blocks() of them).
int launch_partials(const float* d_x, size_t n, double2* d_partials, cudaStream_t s);

// The same with 128-bit loads (d_x 16-byte aligned); with d_copy set, x is
// also copied there; with d_state set, the baseline loop state is started.
int launch_partials_v4(const float* d_x, size_t n, double2* d_partials, float* d_copy,
                       unsigned* d_state, cudaStream_t s);

// One baseline pass in one kernel (the mean of d_part_in formed by every
// CTA): flags and partials alternate between passes; the last pass also
// writes the final flag and the pass count to d_fin_flag / d_fin_passes.
int launch_baseline_pass_v4(float* d_x, size_t n, const double2* d_part_in, double2* d_part_out,
                            const unsigned* d_flag_in, unsigned* d_flag_out, unsigned* d_passes,
                            unsigned* d_fin_flag, unsigned* d_fin_passes, cudaStream_t s);

// launch_running_median without the amplitude array: amplitudes of the
// complex spectrum d_X and their 5/25/125-bin medians in one kernel, then
// the division of d_X by the spliced median in place.
int launch_running_median_spectrum(float* d_X, size_t nbins, double bin_width, float b5,
                                   float b25, void* d_scratch, cudaStream_t s);

// launch_stats(interbinned, first = 0) with 128-bit loads (d_X 16-byte aligned).
int launch_interbin_stats_v4(const float* d_X, size_t nbins, double2* d_partials, double* d_sums,
                             float* d_stat, float scale, cudaStream_t s);

// x[i] -= *d_v.
int launch_sub_scalar(float* d_x, size_t n, const float* d_v, cudaStream_t s);

// Row-batched forms of the prologue stages over `rows` series laid out at
// fixed strides (elements; row r of each buffer starts at base + r *
// stride): the grouped prologue of the search engine.  Each row is computed
// exactly as the single-row launcher computes it.
int launch_partials_rows(const float* d_x, size_t n, size_t x_stride, int rows,
                         double2* d_partials, size_t part_stride, unsigned* d_state,
                         size_t state_stride, cudaStream_t s);
int launch_baseline_pass_rows(float* d_x, size_t n, size_t x_stride, int rows,
                              const double2* d_part_in, double2* d_part_out, size_t part_stride,
                              const unsigned* d_flag_in, unsigned* d_flag_out,
                              unsigned* d_passes, unsigned* d_fin_flag, unsigned* d_fin_passes,
                              size_t flag_stride, cudaStream_t s);
int launch_fill_rows(float* d_x, size_t n, size_t x_stride, int rows, float value,
                     cudaStream_t s);
int launch_running_median_spectrum_rows(float* d_X, size_t x_stride, int rows, size_t nbins,
                                        double bin_width, float b5, float b25, void* d_scratch,
                                        size_t scratch_stride_floats, cudaStream_t s);
int launch_zap_rows(float* d_X, size_t x_stride, int rows, const float* d_freqs,
                    const float* d_widths, float bin_width, size_t nbirdies, size_t nbins,
                    cudaStream_t s);
int launch_interbin_stats_rows(const float* d_X, size_t x_stride, int rows, size_t nbins,
                               double2* d_partials, size_t part_stride, double* d_sums,
                               size_t sums_stride, float* d_stat, size_t stat_stride, float scale,
                               cudaStream_t s);

}  // namespace psx
