// fourierseries.hpp -- frequency-series containers of the drop-in API
// (reference include/data_types/fourierseries.hpp:36-188: FrequencySeries,
// DeviceFourierSeries, DevicePowerSpectrum, HarmonicSums).
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <vector>
#include "utils/exceptions.hpp"

template <class T>
class FrequencySeries {
protected:
    T* data_ptr;
    unsigned int nbins;
    double bin_width;

    FrequencySeries() : data_ptr(nullptr), nbins(0), bin_width(0) {}
    FrequencySeries(unsigned int n, double bw) : data_ptr(nullptr), nbins(n), bin_width(bw) {}

public:
    virtual ~FrequencySeries() {}
    T* get_data() { return data_ptr; }
    void set_data(T* p) { data_ptr = p; }
    double get_bin_width() { return bin_width; }
    void set_bin_width(double bw) { bin_width = bw; }
    unsigned int get_nbins() { return nbins; }
    void set_nbins(unsigned int n) { nbins = n; }
};

template <class T>
class DeviceFrequencySeries : public FrequencySeries<T> {
protected:
    DeviceFrequencySeries(unsigned int n, double bw) : FrequencySeries<T>(n, bw)
    {
        if (cudaMalloc((void**)&this->data_ptr, sizeof(T) * (n ? n : 1)) != cudaSuccess)
            ErrorChecker::throw_error("DeviceFrequencySeries: cudaMalloc failed");
    }

public:
    ~DeviceFrequencySeries() { cudaFree(this->data_ptr); }
    DeviceFrequencySeries(const DeviceFrequencySeries&) = delete;
    DeviceFrequencySeries& operator=(const DeviceFrequencySeries&) = delete;
};

template <class T>
class DeviceFourierSeries : public DeviceFrequencySeries<T> {
public:
    DeviceFourierSeries(unsigned int n, double bw) : DeviceFrequencySeries<T>(n, bw) {}
};

template <class T>
class DevicePowerSpectrum : public DeviceFrequencySeries<T> {
    unsigned int nh;

public:
    DevicePowerSpectrum(unsigned int n, double bw, unsigned int nh_ = 0)
        : DeviceFrequencySeries<T>(n, bw), nh(nh_)
    {
    }
    template <class U>
    DevicePowerSpectrum(FrequencySeries<U>& other, unsigned int nh_ = 0)
        : DeviceFrequencySeries<T>(other.get_nbins(), other.get_bin_width()), nh(nh_)
    {
    }
    unsigned int get_nh() { return nh; }
    void set_nh(unsigned int n) { nh = n; }
};

template <class T>
class HarmonicSums {
    std::vector<DevicePowerSpectrum<T>*> folds;

public:
    HarmonicSums(DevicePowerSpectrum<T>& fold0, unsigned int nfolds)
    {
        for (unsigned int i = 0; i < nfolds; ++i)
            folds.push_back(new DevicePowerSpectrum<T>(fold0, i + 1));
    }
    ~HarmonicSums()
    {
        for (auto* f : folds) delete f;
    }
    HarmonicSums(const HarmonicSums&) = delete;
    HarmonicSums& operator=(const HarmonicSums&) = delete;
    size_t size() { return folds.size(); }
    DevicePowerSpectrum<T>* operator[](int i) { return folds[i]; }
};
