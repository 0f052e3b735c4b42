// dedisperser.hpp -- Dedisperser of the drop-in API (reference
// include/transforms/dedisperser.hpp:13-188, which wraps the external
// dedisp library), over libpeasoup_b200's psx_dedisp_* plan.
//
// dedisperse() keeps the reference's contract: samples [start, end) of the
// filterbank become DispersionTrials of end - start - max_delay samples per
// DM trial in host memory.  dedisperse_device() leaves the block in device
// memory, where the search reads it (the reference copies it to the host and
// each Worker copies one series back per DM trial).
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>
#include "data_types/filterbank.hpp"
#include "data_types/timeseries.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class Dedisperser {
    psx_dedisp_plan* plan;
    Filterbank& filterbank;
    unsigned int num_gpus;
    std::vector<float> dm_list;
    std::vector<int> killmask;
    std::vector<unsigned char> rows;

public:
    Dedisperser(Filterbank& fb, unsigned int num_gpus = 1)
        : plan(nullptr), filterbank(fb), num_gpus(num_gpus)
    {
        killmask.resize((std::size_t)fb.get_nchans(), 1);
        ErrorChecker::check(psx_dedisp_create((std::size_t)fb.get_nchans(), fb.get_tsamp(),
                                              fb.get_fch1(), fb.get_foff(), &plan),
                            "create_plan");
    }
    virtual ~Dedisperser()
    {
        if (plan) psx_dedisp_destroy(plan);
    }
    Dedisperser(const Dedisperser&) = delete;
    Dedisperser& operator=(const Dedisperser&) = delete;

    void set_dm_list(float* dm_list_ptr, unsigned int ndms)
    {
        dm_list.assign(dm_list_ptr, dm_list_ptr + ndms);
        ErrorChecker::check(psx_dedisp_set_dm_list(plan, dm_list.data(), dm_list.size()),
                            "set_dm_list");
    }
    void set_dm_list(std::vector<float> dms) { set_dm_list(dms.data(), (unsigned int)dms.size()); }
    std::vector<float> get_dm_list() { return dm_list; }

    void generate_dm_list(float dm_start, float dm_end, float width, float tolerance)
    {
        ErrorChecker::check(psx_dedisp_generate_dm_list(plan, dm_start, dm_end, width, tolerance),
                            "generate_dm_list");
        dm_list.resize(psx_dedisp_get_dm_count(plan));
        ErrorChecker::check(psx_dedisp_get_dm_list(plan, dm_list.data(), dm_list.size()),
                            "get_dm_list");
    }

    void set_killmask(std::vector<int> killmask_in)
    {
        killmask.swap(killmask_in);
        ErrorChecker::check(psx_dedisp_set_killmask(plan, killmask.data()), "set_killmask");
    }

    // One integer per line, at most nchans lines; a file of another length
    // leaves every channel in, with a warning, as the reference does.
    void set_killmask(std::string filename)
    {
        std::ifstream infile(filename.c_str(), std::ifstream::in | std::ifstream::binary);
        ErrorChecker::check_file_error(infile, filename);
        std::vector<int> km;
        std::string str;
        std::size_t nchans = (std::size_t)filterbank.get_nchans();
        while (!infile.eof() && km.size() < nchans) {
            std::getline(infile, str);
            km.push_back(std::atoi(str.c_str()));
        }
        if (km.size() != nchans) {
            std::cerr << "WARNING: killmask is not the same size as nchans" << std::endl;
            std::cerr << km.size() << " != " << nchans << std::endl;
            km.assign(nchans, 1);
        }
        set_killmask(km);
    }

    std::size_t get_max_delay() { return psx_dedisp_get_max_delay(plan); }
    psx_dedisp_plan* get_plan() { return plan; }

    // Samples [start, end) of the filterbank, read `gulp` rows at a time,
    // dedispersed into d_out (one row of out_pitch floats per DM trial,
    // end - start - max_delay samples each), asynchronously on `stream`.
    void dedisperse_device(float* d_out, std::size_t out_pitch, std::size_t input_start_sample,
                           std::size_t input_end_sample, std::size_t gulp = 0,
                           cudaStream_t stream = 0)
    {
        std::size_t nsamps = input_end_sample - input_start_sample;
        std::size_t row = (std::size_t)filterbank.get_nchans() *
                          (std::size_t)filterbank.get_nbits() / 8;
        rows.resize(nsamps * row);
        std::size_t step = gulp ? gulp : nsamps;
        for (std::size_t pos = 0; pos < nsamps;) {
            std::size_t n = std::min(step, nsamps - pos);
            std::size_t got = filterbank.load_gulp(input_start_sample + pos, n);
            if (got == 0)
                throw std::runtime_error("Failed to read data during dedispersion, 0 samples read.");
            std::memcpy(rows.data() + pos * row, filterbank.get_data(), got * row);
            pos += got;
        }
        ErrorChecker::check(psx_dedisp_execute_host(plan, nsamps, rows.data(),
                                                    (int)filterbank.get_nbits(), d_out, out_pitch,
                                                    0, reinterpret_cast<psx_stream_t>(stream)),
                            "dedisperse");
    }

    void dedisperse(DispersionTrials<float>& trials, std::size_t input_start_sample,
                    std::size_t input_end_sample, std::size_t gulp)
    {
        std::size_t md = get_max_delay();
        std::size_t nsamps = input_end_sample - input_start_sample;
        if (nsamps <= md) ErrorChecker::throw_error("dedisperse: segment shorter than the maximum delay");
        std::size_t nout = nsamps - md;
        std::size_t pitch = (nout + 3) / 4 * 4;
        trials.resize(nout, dm_list);
        float* d_out = nullptr;
        if (cudaMalloc((void**)&d_out, sizeof(float) * pitch * dm_list.size()) != cudaSuccess)
            ErrorChecker::throw_error("dedisperse: cudaMalloc failed");
        try {
            dedisperse_device(d_out, pitch, input_start_sample, input_end_sample, gulp);
            cudaError_t e = cudaMemcpy2D(trials.get_data_ptr(), nout * sizeof(float), d_out,
                                         pitch * sizeof(float), nout * sizeof(float),
                                         dm_list.size(), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) ErrorChecker::throw_error(std::string("dedisperse: ") +
                                                            cudaGetErrorString(e));
        } catch (...) {
            cudaFree(d_out);
            throw;
        }
        cudaFree(d_out);
    }
};
