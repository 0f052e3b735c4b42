// resampler.hpp -- TimeDomainResampler of the drop-in API (reference
// include/transforms/resampler.hpp:7-34) over psx_resample/psx_resampleII.
#pragma once
#include "data_types/timeseries.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class TimeDomainResampler {
    psx_stream_t stream;

public:
    explicit TimeDomainResampler(psx_stream_t s = nullptr) : stream(s) {}

    void resample(DeviceTimeSeries<float>& input, DeviceTimeSeries<float>& output,
                  unsigned int size, float acc)
    {
        ErrorChecker::check(psx_resample(input.get_data(), output.get_data(), size, acc,
                                         input.get_tsamp(), stream),
                            "TimeDomainResampler::resample");
    }

    void resampleII(DeviceTimeSeries<float>& input, DeviceTimeSeries<float>& output,
                    unsigned int size, float acc)
    {
        ErrorChecker::check(psx_resampleII(input.get_data(), output.get_data(), size, acc,
                                           input.get_tsamp(), stream),
                            "TimeDomainResampler::resampleII");
    }
};
