// stats.hpp -- the stats namespace of the drop-in API (reference
// include/utils/stats.hpp:6-43): mean/rms/std of a device array
// (synchronous) and the in-place normalisation (asynchronous).
#pragma once
#include <cmath>
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

namespace stats {

template <class T>
float rms(T* ptr, unsigned int nsamps, unsigned int first_samp = 0)
{
    float m, r, s;
    ErrorChecker::check(psx_stats(ptr, nsamps, first_samp, &m, &r, &s, nullptr), "stats::rms");
    return r;
}

template <class T>
float mean(T* ptr, unsigned int nsamps, unsigned int first_samp = 0)
{
    float m, r, s;
    ErrorChecker::check(psx_stats(ptr, nsamps, first_samp, &m, &r, &s, nullptr), "stats::mean");
    return m;
}

inline float std(float mean_, float rms_) { return std::sqrt(rms_ * rms_ - mean_ * mean_); }

template <class T>
void stats(T* ptr, unsigned int nsamps, float* mean_, float* rms_, float* std_,
           unsigned int first_samp = 0)
{
    ErrorChecker::check(psx_stats(ptr, nsamps, first_samp, mean_, rms_, std_, nullptr),
                        "stats::stats");
}

inline void normalise(float* ptr, float mean_, float std_, unsigned int size,
                      psx_stream_t stream = nullptr)
{
    ErrorChecker::check(psx_normalise(ptr, mean_, std_, size, stream), "stats::normalise");
}

}  // namespace stats
