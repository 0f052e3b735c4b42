// utils.hpp -- AccelerationPlan of the drop-in API (reference
// include/utils/utils.hpp:143-233): the per-DM acceleration trial list,
// computed by libpeasoup_b200 with the reference's float arithmetic.
#pragma once
#include <cstddef>
#include <vector>
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class AccelerationPlan {
    float acc_lo, acc_hi, tol, pulse_width;
    std::size_t nsamps;
    float tsamp, cfreq, ch_bw;

public:
    AccelerationPlan(float acc_lo, float acc_hi, float tol, float pulse_width,
                     std::size_t nsamps, float tsamp, float cfreq, float ch_bw)
        : acc_lo(acc_lo), acc_hi(acc_hi), tol(tol), pulse_width(pulse_width),
          nsamps(nsamps), tsamp(tsamp), cfreq(cfreq), ch_bw(ch_bw)
    {
    }

    void generate_accel_list(float dm, float cdm, std::vector<float>& acc_list) const
    {
        std::size_t n = 0;
        ErrorChecker::check(psx_accel_list(acc_lo, acc_hi, tol, pulse_width, nsamps, tsamp,
                                           cfreq, ch_bw, dm, cdm, nullptr, 0, &n),
                            "AccelerationPlan::generate_accel_list");
        acc_list.resize(n);
        ErrorChecker::check(psx_accel_list(acc_lo, acc_hi, tol, pulse_width, nsamps, tsamp,
                                           cfreq, ch_bw, dm, cdm, acc_list.data(), n, &n),
                            "AccelerationPlan::generate_accel_list");
    }
};
