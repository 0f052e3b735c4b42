// timeseries.hpp -- time-series containers of the drop-in API (reference
// include/data_types/timeseries.hpp:58-372: TimeSeries, DeviceTimeSeries,
// ReusableDeviceTimeSeries, DedispersedTimeSeries).  Device buffers are
// plain cudaMalloc allocations owned by the object; the operations call
// libpeasoup_b200 on the legacy default stream, asynchronously.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <string>
#include <type_traits>
#include <vector>
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

template <class T>
class TimeSeries {
protected:
    T* data_ptr;
    std::size_t nsamps;
    float tsamp;

public:
    TimeSeries() : data_ptr(nullptr), nsamps(0), tsamp(0.0f) {}
    explicit TimeSeries(std::size_t n) : data_ptr(nullptr), nsamps(n), tsamp(0.0f) {}
    TimeSeries(T* p, std::size_t n, float ts) : data_ptr(p), nsamps(n), tsamp(ts) {}
    virtual ~TimeSeries() {}
    T* get_data() { return data_ptr; }
    void set_data(T* p) { data_ptr = p; }
    std::size_t get_nsamps() { return nsamps; }
    void set_nsamps(std::size_t n) { nsamps = n; }
    float get_tsamp() { return tsamp; }
    void set_tsamp(float ts) { tsamp = ts; }
};

template <class T>
class DedispersedTimeSeries : public TimeSeries<T> {
    float dm;

public:
    DedispersedTimeSeries() : TimeSeries<T>(), dm(0.0f) {}
    DedispersedTimeSeries(T* p, std::size_t n, float ts, float dm_)
        : TimeSeries<T>(p, n, ts), dm(dm_)
    {
    }
    float get_dm() { return dm; }
    void set_dm(float d) { dm = d; }
};

template <class OnDeviceType>
class DeviceTimeSeries : public TimeSeries<OnDeviceType> {
    static_assert(sizeof(OnDeviceType) == 4, "device series are float");

public:
    explicit DeviceTimeSeries(std::size_t n) : TimeSeries<OnDeviceType>(n)
    {
        if (cudaMalloc((void**)&this->data_ptr, sizeof(OnDeviceType) * (n ? n : 1)) != cudaSuccess)
            ErrorChecker::throw_error("DeviceTimeSeries: cudaMalloc failed");
    }
    ~DeviceTimeSeries() { cudaFree(this->data_ptr); }
    DeviceTimeSeries(const DeviceTimeSeries&) = delete;
    DeviceTimeSeries& operator=(const DeviceTimeSeries&) = delete;

    // Iterative mean removal over the first nsamps samples (all if 0).
    void remove_baseline(std::size_t nsamps = 0)
    {
        if (nsamps == 0) nsamps = this->nsamps;
        ErrorChecker::check(psx_remove_baseline((float*)this->data_ptr, nsamps, nullptr, nullptr),
                            "DeviceTimeSeries::remove_baseline");
    }

    void fill(std::size_t start, std::size_t end, OnDeviceType value)
    {
        if (end > this->nsamps)
            ErrorChecker::throw_error("DeviceTimeSeries::fill bad end value requested");
        if (end > start)
            ErrorChecker::check(psx_fill((float*)this->data_ptr + start, end - start, (float)value,
                                         nullptr),
                                "DeviceTimeSeries::fill");
    }
};

// Reusable device series with host->device copy (float or uint8 host data).
template <class OnDeviceType, class OnHostType>
class ReusableDeviceTimeSeries : public DeviceTimeSeries<OnDeviceType> {
    void* staging;

public:
    explicit ReusableDeviceTimeSeries(std::size_t n) : DeviceTimeSeries<OnDeviceType>(n), staging(nullptr)
    {
        if (!std::is_same<OnHostType, OnDeviceType>::value &&
            cudaMalloc(&staging, sizeof(OnHostType) * (n ? n : 1)) != cudaSuccess)
            ErrorChecker::throw_error("ReusableDeviceTimeSeries: cudaMalloc failed");
    }
    ~ReusableDeviceTimeSeries()
    {
        if (staging) cudaFree(staging);
    }

    void copy_from_host(TimeSeries<OnHostType>& host)
    {
        const std::size_t n = host.get_nsamps() < this->nsamps ? host.get_nsamps() : this->nsamps;
        this->tsamp = host.get_tsamp();
        if constexpr (std::is_same<OnHostType, OnDeviceType>::value) {
            if (cudaMemcpy(this->data_ptr, host.get_data(), sizeof(OnHostType) * n,
                           cudaMemcpyHostToDevice) != cudaSuccess)
                ErrorChecker::throw_error("copy_from_host: cudaMemcpy failed");
        } else {
            // the reference converts after the copy (conversion_kernel,
            // src/kernels.cu:1171-1200) for its 8-bit host types only
            static_assert(std::is_same<OnDeviceType, float>::value && sizeof(OnHostType) == 1 &&
                              std::is_integral<OnHostType>::value,
                          "host series are float (copied) or 8-bit integers (converted)");
            if (cudaMemcpy(staging, host.get_data(), n, cudaMemcpyHostToDevice) != cudaSuccess)
                ErrorChecker::throw_error("copy_from_host: cudaMemcpy failed");
            int rc;
            if (std::is_signed<OnHostType>::value)
                rc = psx_convert_i8_f32((const int8_t*)staging, (float*)this->data_ptr, n,
                                        nullptr);
            else
                rc = psx_convert_u8_f32((const uint8_t*)staging, (float*)this->data_ptr, n,
                                        nullptr);
            ErrorChecker::check(rc, "copy_from_host");
        }
    }
};

// Host-side block of dedispersed series, one per DM trial (reference
// include/data_types/timeseries.hpp:383-505, without the file writers).
template <class T>
class DispersionTrials {
    std::vector<T> data;
    std::vector<float> dm_list;
    std::size_t nsamps;
    float tsamp;

public:
    explicit DispersionTrials(float ts) : nsamps(0), tsamp(ts) {}
    void resize(std::size_t n, const std::vector<float>& dms)
    {
        dm_list = dms;
        nsamps = n;
        data.resize(n * dms.size());
    }
    std::size_t get_count() const { return dm_list.size(); }
    std::size_t get_nsamps() const { return nsamps; }
    float get_tsamp() const { return tsamp; }
    T* get_data_ptr() { return data.data(); }
    const std::vector<float>& get_dm_list() const { return dm_list; }
    void get_idx(std::size_t idx, DedispersedTimeSeries<T>& tim, std::size_t = 0)
    {
        tim.set_data(data.data() + idx * nsamps);
        tim.set_dm(dm_list[idx]);
        tim.set_nsamps(nsamps);
        tim.set_tsamp(tsamp);
    }
};
