// psx_fft.cuh -- internal cuFFT plan wrapper.
#pragma once
#include <cufft.h>
#include <cuda_runtime.h>
#include <cstddef>
#include "psx_fft_cb.h"

namespace psx {

bool fft_size_supported(size_t n);

// Internal plan kind (beside PSX_FFT_R2C / PSX_FFT_C2R): forward complex
// transform of length n, distances in complex elements.
constexpr int kFftC2C = 100;

struct FftPlan {
    cufftHandle h = 0;
    bool have = false;
    bool callback = false;
    size_t n = 0;
    long long batch = 0;
    int kind = 0;
    size_t work_bytes = 0;
    void* d_cbinfo = nullptr;
    psx_resample_cb_info host_info{};

    // Batched plan of `batch` transforms with the given input/output
    // distances (0 = packed).  With resample_callback the R2C input is read
    // through the resample load callback (set_resample selects the series
    // and the per-trial factors).
    int create(size_t n, long long batch, int kind, size_t in_dist, size_t out_dist,
               bool resample_callback);
    void destroy();
    int set_resample(const float* d_series, const double* d_ktab, cudaStream_t s);
    int exec(const void* in, void* out, cudaStream_t s);
    ~FftPlan() { destroy(); }
};

}  // namespace psx
