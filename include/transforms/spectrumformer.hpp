// spectrumformer.hpp -- SpectrumFormer of the drop-in API (reference
// include/transforms/spectrumformer.hpp:6-24) over psx_form_power_series.
#pragma once
#include <cufft.h>
#include "data_types/fourierseries.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class SpectrumFormer {
    psx_stream_t stream;

public:
    explicit SpectrumFormer(psx_stream_t s = nullptr) : stream(s) {}

    void form_interpolated(DeviceFourierSeries<cufftComplex>& input,
                           DevicePowerSpectrum<float>& output)
    {
        ErrorChecker::check(psx_form_power_series((const float*)input.get_data(), output.get_data(),
                                                  input.get_nbins(), 1, stream),
                            "SpectrumFormer::form_interpolated");
    }

    void form(DeviceFourierSeries<cufftComplex>& input, DevicePowerSpectrum<float>& output)
    {
        ErrorChecker::check(psx_form_power_series((const float*)input.get_data(), output.get_data(),
                                                  input.get_nbins(), 0, stream),
                            "SpectrumFormer::form");
    }
};
