// psx_host.h -- host-side search logic shared by the C ABI and the engine.
#pragma once
#include <cstddef>
#include <vector>
#include "peasoup_b200.h"

namespace psx {

std::vector<float> accel_list(float acc_lo, float acc_hi, float tol, float pulse_width,
                              size_t nsamps, float tsamp, float cfreq, float ch_bw, float dm,
                              float cdm);

void peak_range(unsigned nbins, double bin_width, int nh, float min_freq, float max_freq,
                int* start, int* end, float* factor);

size_t unique_peaks(const int* idx, const float* snr, size_t count, int min_gap, int* oi,
                    float* os);

size_t distill(int kind, psx_candidate* c, size_t n, float tol, float max_harm, float tobs,
               int keep_related, int fractional, int* nassoc);

}  // namespace psx
