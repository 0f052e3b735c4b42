// psx_fft.cuh -- internal cuFFT plan wrapper.
#pragma once
#include <cufft.h>
#include <cuda_runtime.h>
#include <cstddef>

namespace psx {

bool fft_size_supported(size_t n);

// Internal plan kind (beside PSX_FFT_R2C / PSX_FFT_C2R): forward complex
// transform of length n, distances in complex elements.
constexpr int kFftC2C = 100;

struct FftPlan {
    cufftHandle h = 0;
    bool have = false;
    size_t n = 0;
    long long batch = 0;
    int kind = 0;
    size_t work_bytes = 0;

    // Batched plan of `batch` transforms with the given input/output
    // distances (0 = packed).
    int create(size_t n, long long batch, int kind, size_t in_dist, size_t out_dist);
    void destroy();
    int exec(const void* in, void* out, cudaStream_t s);
    // complex plans only: direction CUFFT_FORWARD (-1) or CUFFT_INVERSE (+1)
    int exec_c2c(const void* in, void* out, int direction, cudaStream_t s);
    ~FftPlan() { destroy(); }
};

}  // namespace psx
