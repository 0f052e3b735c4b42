// spectrumnormaliser.hpp -- the normalisation step of the search loop as a
// transform.  The reference has no class of this name: its loop calls
// stats::normalise(pspec, mean*size, std*size, size/2+1)
// (src/pipeline_multi.cu:271).  SpectrumNormaliser holds the two constants
// formed the same way (float products with the transform length).
#pragma once
#include "data_types/fourierseries.hpp"
#include "utils/stats.hpp"

class SpectrumNormaliser {
    float mean_n, std_n;

public:
    SpectrumNormaliser(float mean, float std_, unsigned int fft_size)
        : mean_n(mean * fft_size), std_n(std_ * fft_size)
    {
    }
    void normalise(DevicePowerSpectrum<float>& pspec, psx_stream_t stream = nullptr)
    {
        stats::normalise(pspec.get_data(), mean_n, std_n, pspec.get_nbins(), stream);
    }
};
