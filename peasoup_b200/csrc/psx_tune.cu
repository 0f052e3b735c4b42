// psx_tune.cu -- the autotuner of the batched search: trials per launch
// group and the harmonic kernel's tile shape, chosen by timing the real
// engine on seeded synthetic noise of the caller's transform length.
//
// The reference has one fixed schedule (one trial per launch sequence,
// src/pipeline_multi.cu:244-290), so nothing here replaces a reference
// function.  What the tuner picks changes only how the work is grouped,
// never a result: every shape sums in the reference's order, and every
// batch runs the same per-trial arithmetic.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>
#include "psx_common.cuh"
#include "psx_host.h"

namespace psx {
namespace {

// Seeded white noise: the SplitMix64 output function of (seed, index) gives
// two 24-bit uniforms, then the Box-Muller transform.  Only its statistics matter to the tuner (how
// often a bin crosses the threshold), not its exact values.
__global__ void __launch_bounds__(256) k_tune_noise(float* __restrict__ x, size_t n,
                                                    unsigned long long seed)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const float u1 = ((unsigned)(z >> 40) + 0.5f) * (1.0f / 16777216.0f);
        const float u2 = ((unsigned)(z & 0xffffffu) + 0.5f) * (1.0f / 16777216.0f);
        x[i] = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
    }
}

struct Timing {
    int batch, shape;
    double ms;  // wall-clock milliseconds per DM trial
};

}  // namespace
}  // namespace psx

using namespace psx;

extern "C" int psx_autotune(psx_search_config* cfg, const int* h_batches, int nbatch, int reps,
                            int max_trials, double* h_ms)
{
    clear_error();
    if (!cfg || !h_batches || nbatch < 1 || reps < 1 || max_trials < 1) {
        set_error("autotune: bad arguments");
        return PSX_ERR_INVALID;
    }
    for (int i = 0; i < nbatch; ++i)
        if (h_batches[i] < 1 || h_batches[i] > 1024) {
            set_error("autotune: batch %d outside 1..1024", h_batches[i]);
            return PSX_ERR_INVALID;
        }
    psx_search_config base = *cfg;
    base.mode = PSX_MODE_BATCHED;
    base.use_fft_callback = 0;
    // Narrow the acceleration range around its middle when the DM-0 list is
    // longer than max_trials: the per-trial cost does not depend on where
    // the trials lie, and the tuner must stay short at 2^27.
    const std::vector<float> full =
        accel_list(base.acc_lo, base.acc_hi, base.acc_tol, base.acc_pulse_width, base.fft_size,
                   base.tsamp, base.cfreq_hz, base.ch_bw_hz, 0.0f, base.cdm);
    if ((int)full.size() > max_trials && base.acc_hi > base.acc_lo) {
        const double f = (double)max_trials / (double)full.size();
        const double mid = 0.5 * ((double)base.acc_lo + base.acc_hi);
        const double half = 0.5 * ((double)base.acc_hi - base.acc_lo) * f;
        base.acc_lo = (float)(mid - half);
        base.acc_hi = (float)(mid + half);
    }
    size_t free_b = 0, total_b = 0;
    PSX_CUDA(cudaMemGetInfo(&free_b, &total_b));

    const size_t N = base.fft_size;
    float* d_x = nullptr;
    PSX_CUDA(cudaMalloc(&d_x, sizeof(float) * N));
    k_tune_noise<<<grid_for(N, 256), 256>>>(d_x, N, 0x5eedull);
    int rc = launch_status("autotune noise kernel");
    if (rc == PSX_OK) rc = cuda_status(cudaDeviceSynchronize(), "autotune noise");

    std::vector<const float*> series((size_t)reps + 1, d_x);
    std::vector<float> dms((size_t)reps + 1, 0.0f);
    std::vector<psx_candidate> out((size_t)1 << 20);
    std::vector<Timing> timings;
    for (int bi = 0; bi < nbatch && rc == PSX_OK; ++bi) {
        for (int shape = 1; shape <= PSX_HARM_SHAPES && rc == PSX_OK; ++shape) {
            psx_search_config c = base;
            c.batch = h_batches[bi];
            c.harm_shape = shape;
            double ms = -1.0;
            if (psx_search_footprint(&c) < free_b / 10 * 8) {
                psx_search* s = nullptr;
                rc = psx_search_create(&c, &s);
                if (rc == PSX_ERR_INVALID) {  // a shape this batch cannot use: skip it
                    clear_error();
                    rc = PSX_OK;
                } else if (rc == PSX_OK) {
                    size_t n = 0;
                    // one DM to warm up (plans, graph capture), then `reps`
                    // DMs through the pipelined block call, timed on the host
                    rc = psx_search_dm(s, d_x, N, 1, 0.0f, 0, PSX_OUT_TRIAL, out.data(), nullptr,
                                       nullptr, out.size(), &n);
                    if (rc == PSX_ERR_OVERFLOW) rc = PSX_OK;
                    const auto t0 = std::chrono::steady_clock::now();
                    if (rc == PSX_OK)
                        rc = psx_search_block(s, series.data(), N, 1, dms.data(), nullptr, reps,
                                              PSX_OUT_TRIAL, out.data(), nullptr, nullptr, nullptr,
                                              out.size(), &n);
                    if (rc == PSX_ERR_OVERFLOW) rc = PSX_OK;
                    const auto t1 = std::chrono::steady_clock::now();
                    ms = std::chrono::duration<double, std::milli>(t1 - t0).count() / reps;
                    psx_search_destroy(s);
                }
            }
            if (h_ms) h_ms[bi * PSX_HARM_SHAPES + (shape - 1)] = ms;
            if (ms > 0.0) timings.push_back({h_batches[bi], shape, ms});
        }
    }
    cudaFree(d_x);
    if (rc != PSX_OK) return rc;
    if (timings.empty()) {
        set_error("autotune: no candidate fits in device memory");
        return PSX_ERR_ALLOC;
    }
    const Timing best = *std::min_element(
        timings.begin(), timings.end(), [](const Timing& a, const Timing& b) { return a.ms < b.ms; });
    cfg->batch = best.batch;
    cfg->harm_shape = best.shape;
    return PSX_OK;
}
