// psx_fft_cb.h -- caller-info block of the resample load callback.
#pragma once
#include <stdint.h>

struct psx_resample_cb_info {
    const float* series;      // dereddened series, N floats
    const double* ktab;       // accel factor of each trial of the batch
    unsigned long long n;     // N = 2^shift or 3*2^shift
    double size;              // (double)N
    unsigned shift;
    unsigned three;           // 1 when N = 3*2^shift
};
