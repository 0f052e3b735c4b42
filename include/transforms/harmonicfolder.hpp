// harmonicfolder.hpp -- HarmonicFolder of the drop-in API (reference
// include/transforms/harmonicfolder.hpp:8-45).  The output pointers are
// passed to the kernel by value; nothing is copied to the device per call.
#pragma once
#include <vector>
#include "data_types/fourierseries.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class HarmonicFolder {
    HarmonicSums<float>& sums;
    psx_stream_t stream;

public:
    explicit HarmonicFolder(HarmonicSums<float>& s, psx_stream_t st = nullptr) : sums(s), stream(st) {}

    void fold(DevicePowerSpectrum<float>& fold0)
    {
        std::vector<float*> ptrs(sums.size());
        for (size_t i = 0; i < sums.size(); ++i) ptrs[i] = sums[(int)i]->get_data();
        ErrorChecker::check(psx_harmonic_sum(fold0.get_data(), ptrs.data(), fold0.get_nbins(),
                                             (int)sums.size(), stream),
                            "HarmonicFolder::fold");
    }
};
