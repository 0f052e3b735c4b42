// filterbank.hpp -- filterbank input of the drop-in API (reference
// include/data_types/filterbank.hpp:25-361: Filterbank, SigprocFilterbank),
// reading through libpeasoup_b200 (psx_sigproc_read_header,
// psx_sigproc_read).  Metadata keeps the reference's types: tsamp, fch1 and
// foff are float; the getters of nchans and nbits return float as the
// reference's do.
#pragma once
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>
#include "data_types/header.hpp"
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class Filterbank {
protected:
    unsigned char* data;
    unsigned int total_nsamps;
    unsigned int nchans;
    unsigned char nbits;
    float fch1;
    float foff;
    float tsamp;
    unsigned long start_sample;
    unsigned long end_sample;
    unsigned long effective_nsamps;

    Filterbank()
        : data(nullptr), total_nsamps(0), nchans(0), nbits(0), fch1(0), foff(0), tsamp(0),
          start_sample(0), end_sample(0), effective_nsamps(0)
    {
    }

public:
    virtual ~Filterbank() {}
    virtual float get_tsamp() { return tsamp; }
    virtual void set_tsamp(float t) { tsamp = t; }
    virtual float get_foff() { return foff; }
    virtual void set_foff(float f) { foff = f; }
    virtual float get_fch1() { return fch1; }
    virtual void set_fch1(float f) { fch1 = f; }
    virtual float get_nchans() { return nchans; }
    virtual void set_nchans(unsigned int n) { nchans = n; }
    virtual unsigned int get_total_nsamps() { return total_nsamps; }
    virtual void set_total_nsamps(unsigned int n) { total_nsamps = n; }
    virtual float get_nbits() { return nbits; }
    virtual void set_nbits(unsigned char b) { nbits = b; }
    virtual unsigned char* get_data() { return data; }
    virtual void set_data(unsigned char* d) { data = d; }
    virtual unsigned long get_start_sample() { return start_sample; }
    virtual unsigned long get_end_sample() { return end_sample; }
    virtual unsigned long get_effective_nsamps() { return effective_nsamps; }
    virtual std::size_t load_gulp(std::size_t, std::size_t) { return 0; }
    virtual double get_segment_pepoch() { return -1; }

    // Centre frequency (MHz), in float as the reference computes it.
    virtual float get_cfreq()
    {
        if (foff < 0) return fch1 + foff * nchans / 2;
        return fch1 - foff * nchans / 2;
    }
};

class SigprocFilterbank : public Filterbank {
public:
    unsigned int size;  // transform length, for get_segment_pepoch

    // Opens `filename`, reads its header and selects the segment
    // [segment_start_sample, + segment_nsamples); 0 samples, or a segment
    // past the end, runs to the end of the file with a warning.
    SigprocFilterbank(std::string filename, std::size_t segment_start_sample,
                      std::size_t segment_nsamples)
        : size(0), path(filename)
    {
        ErrorChecker::check(psx_sigproc_read_header(path.c_str(), &raw), "SigprocFilterbank");
        header.from_c(raw);
        total_nsamps = (unsigned int)header.nsamples;
        nchans = (unsigned int)header.nchans;
        tsamp = (float)header.tsamp;
        nbits = (unsigned char)header.nbits;
        fch1 = (float)header.fch1;
        foff = (float)header.foff;
        start_sample = segment_start_sample;
        if (segment_start_sample > total_nsamps) ErrorChecker::throw_error("Invalid start sample provided.");
        if (segment_nsamples == 0 || segment_start_sample + segment_nsamples > total_nsamps) {
            std::cerr << "Warning: Requested segment exceeds total samples available in filterbank. "
                      << "Adjusting to last available sample.\n";
            end_sample = total_nsamps;
        } else {
            end_sample = segment_start_sample + segment_nsamples;
        }
        effective_nsamps = end_sample - start_sample;
    }

    // Reads up to gulp_nsamples rows from gulp_start_sample into the
    // object's buffer (get_data()); returns the rows read.
    std::size_t load_gulp(std::size_t gulp_start_sample, std::size_t gulp_nsamples) override
    {
        std::size_t row = (std::size_t)raw.nchans * (std::size_t)raw.nbits / 8;
        buffer.resize(gulp_nsamples * row);
        std::size_t got = 0;
        ErrorChecker::check(psx_sigproc_read(path.c_str(), &raw, gulp_start_sample, gulp_nsamples,
                                             buffer.data(), &got),
                            "load_gulp");
        buffer.resize(got * row);
        set_data(buffer.data());
        return got;
    }

    SigprocHeader get_header() { return header; }
    const psx_sigproc_header& get_c_header() const { return raw; }
    const std::string& get_filename() const { return path; }

    double get_segment_pepoch() override
    {
        double start_time = start_sample * tsamp / 86400.0;
        double end_time = size * tsamp / 86400.0;
        double tstart_updated = header.tstart + start_time;
        return tstart_updated + 0.5 * end_time;
    }

private:
    std::string path;
    SigprocHeader header;
    psx_sigproc_header raw;
    std::vector<unsigned char> buffer;
};
