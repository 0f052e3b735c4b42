// dereddener.hpp -- Dereddener of the drop-in API (reference
// include/transforms/dereddener.hpp:10-68): spliced 5/25/125-bin running
// median and the division of the complex spectrum by it.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include "data_types/fourierseries.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class Dereddener {
    unsigned int size;
    float* median;
    void* scratch;
    psx_stream_t stream;

public:
    explicit Dereddener(unsigned int n, psx_stream_t s = nullptr)
        : size(n), median(nullptr), scratch(nullptr), stream(s)
    {
        if (cudaMalloc((void**)&median, sizeof(float) * (n ? n : 1)) != cudaSuccess ||
            cudaMalloc(&scratch, psx_running_median_scratch_bytes(n)) != cudaSuccess)
            ErrorChecker::throw_error("Dereddener: cudaMalloc failed");
    }
    virtual ~Dereddener()
    {
        cudaFree(median);
        cudaFree(scratch);
    }
    Dereddener(const Dereddener&) = delete;
    Dereddener& operator=(const Dereddener&) = delete;

    void calculate_median(DevicePowerSpectrum<float>& powers, float boundary_5_freq = 0.05,
                          float boundary_25_freq = 0.5)
    {
        if (powers.get_nbins() != size)
            ErrorChecker::throw_error("Bad data length given to running_median()");
        ErrorChecker::check(psx_running_median(powers.get_data(), size, powers.get_bin_width(),
                                               boundary_5_freq, boundary_25_freq, median, scratch,
                                               stream),
                            "Dereddener::calculate_median");
    }

    void deredden(DeviceFourierSeries<cufftComplex>& spectrum)
    {
        ErrorChecker::check(psx_divide_c_by_f((float*)spectrum.get_data(), median,
                                              spectrum.get_nbins(), stream),
                            "Dereddener::deredden");
    }

    float* get_median() { return median; }
};
