// peakfinder.hpp -- PeakFinder of the drop-in API (reference
// include/transforms/peakfinder.hpp:11-95): threshold, order-preserving
// compaction on the device, min-gap clustering and frequency assignment.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "data_types/candidates.hpp"
#include "data_types/fourierseries.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class PeakFinder {
    float threshold, min_freq, max_freq;
    int min_gap;
    int cap;
    int* d_idx;
    float* d_val;
    std::vector<int> idx, pidx;
    std::vector<float> val, psnr, pfreq;
    psx_stream_t stream;

    void alloc(int n)
    {
        if (d_idx) cudaFree(d_idx);
        if (d_val) cudaFree(d_val);
        cap = n;
        if (cudaMalloc((void**)&d_idx, sizeof(int) * cap) != cudaSuccess ||
            cudaMalloc((void**)&d_val, sizeof(float) * cap) != cudaSuccess)
            ErrorChecker::throw_error("PeakFinder: cudaMalloc failed");
    }

public:
    PeakFinder(float threshold_, float min_freq_, float max_freq_, unsigned int size,
               int min_gap_ = 30, psx_stream_t s = nullptr)
        : threshold(threshold_), min_freq(min_freq_), max_freq(max_freq_), min_gap(min_gap_),
          cap(0), d_idx(nullptr), d_val(nullptr), stream(s)
    {
        alloc(size > 1024 ? (int)size : 1024);
    }
    ~PeakFinder()
    {
        cudaFree(d_idx);
        cudaFree(d_val);
    }
    PeakFinder(const PeakFinder&) = delete;
    PeakFinder& operator=(const PeakFinder&) = delete;

    void find_candidates(HarmonicSums<float>& sums, SpectrumCandidates& cands)
    {
        for (size_t i = 0; i < sums.size(); ++i) find_candidates(*sums[(int)i], cands);
    }

    void find_candidates(DevicePowerSpectrum<float>& pspec, SpectrumCandidates& cands)
    {
        int start, end;
        float factor;
        ErrorChecker::check(psx_peak_range(pspec.get_nbins(), pspec.get_bin_width(),
                                           (int)pspec.get_nh(), min_freq, max_freq, &start, &end,
                                           &factor),
                            "PeakFinder::find_candidates");
        int count = 0;
        int rc = psx_find_peaks(pspec.get_data(), end, start, threshold, d_idx, d_val, cap, &count,
                                stream);
        if (rc == PSX_ERR_OVERFLOW) {
            alloc(count + count / 4 + 1024);
            rc = psx_find_peaks(pspec.get_data(), end, start, threshold, d_idx, d_val, cap, &count,
                                stream);
        }
        ErrorChecker::check(rc, "PeakFinder::find_candidates");
        if (count == 0) return;
        idx.resize(count);
        val.resize(count);
        cudaMemcpy(idx.data(), d_idx, sizeof(int) * count, cudaMemcpyDeviceToHost);
        cudaMemcpy(val.data(), d_val, sizeof(float) * count, cudaMemcpyDeviceToHost);
        pidx.resize(count);
        psnr.resize(count);
        const size_t np =
            psx_identify_unique_peaks(idx.data(), val.data(), count, min_gap, pidx.data(), psnr.data());
        pfreq.resize(np);
        for (size_t i = 0; i < np; ++i) pfreq[i] = pidx[i] * factor;
        cands.append(psnr.data(), pfreq.data(), (int)pspec.get_nh(), (int)np);
    }
};
