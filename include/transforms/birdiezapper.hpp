// birdiezapper.hpp -- Zapper of the drop-in API (reference
// include/transforms/birdiezapper.hpp:11-73): a zap list of "freq width"
// lines; zap() sets the affected bins of a complex spectrum to 1+0i.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <string>
#include <vector>
#include "data_types/fourierseries.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class Zapper {
    std::vector<float> birdies, widths;
    float* d_birdies;
    float* d_widths;
    psx_stream_t stream;

    void upload()
    {
        if (d_birdies) cudaFree(d_birdies);
        if (d_widths) cudaFree(d_widths);
        d_birdies = d_widths = nullptr;
        const size_t n = birdies.size() ? birdies.size() : 1;
        if (cudaMalloc((void**)&d_birdies, sizeof(float) * n) != cudaSuccess ||
            cudaMalloc((void**)&d_widths, sizeof(float) * n) != cudaSuccess)
            ErrorChecker::throw_error("Zapper: cudaMalloc failed");
        if (!birdies.empty()) {
            cudaMemcpy(d_birdies, birdies.data(), sizeof(float) * birdies.size(), cudaMemcpyHostToDevice);
            cudaMemcpy(d_widths, widths.data(), sizeof(float) * widths.size(), cudaMemcpyHostToDevice);
        }
    }

public:
    explicit Zapper(const std::string& zaplist, psx_stream_t s = nullptr)
        : d_birdies(nullptr), d_widths(nullptr), stream(s)
    {
        append_from_file(zaplist);
    }
    ~Zapper()
    {
        if (d_birdies) cudaFree(d_birdies);
        if (d_widths) cudaFree(d_widths);
    }
    Zapper(const Zapper&) = delete;
    Zapper& operator=(const Zapper&) = delete;

    void append_from_file(const std::string& zaplist)
    {
        size_t n = 0;
        ErrorChecker::check(psx_read_zaplist(zaplist.c_str(), nullptr, nullptr, 0, &n), "Zapper");
        std::vector<float> f(n ? n : 1), w(n ? n : 1);
        ErrorChecker::check(psx_read_zaplist(zaplist.c_str(), f.data(), w.data(), n, &n), "Zapper");
        birdies.insert(birdies.end(), f.begin(), f.begin() + n);
        widths.insert(widths.end(), w.begin(), w.begin() + n);
        upload();
    }

    const std::vector<float>& get_birdies() const { return birdies; }
    const std::vector<float>& get_widths() const { return widths; }

    void zap(DeviceFourierSeries<cufftComplex>& fseries)
    {
        zap(fseries.get_data(), (float)fseries.get_bin_width(), fseries.get_nbins());
    }

    void zap(cufftComplex* fseries, float bin_width, unsigned int nbins)
    {
        ErrorChecker::check(psx_zap_birdies((float*)fseries, d_birdies, d_widths, bin_width,
                                            birdies.size(), nbins, stream),
                            "Zapper::zap");
    }
};
