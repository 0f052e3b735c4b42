// header.hpp -- SIGPROC header of the drop-in API (reference
// include/data_types/header.hpp:171-212 SigprocHeader, :339-403
// read_header), parsed by libpeasoup_b200 (psx_sigproc_parse_header).
#pragma once
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include "peasoup_b200.h"
#include "utils/exceptions.hpp"

class SigprocHeader {
public:
    std::string source_name;
    std::string rawdatafile;
    double az_start, za_start, src_raj, src_dej, tstart, tsamp, period, fch1, foff;
    int nchans, telescope_id, machine_id, data_type, ibeam, nbeams, nbits;
    int barycentric, pulsarcentric, nbins, nsamples, nifs, npuls;
    double refdm;
    unsigned char signed_data;
    unsigned int size;  // header bytes

    SigprocHeader()
        : az_start(0), za_start(0), src_raj(0), src_dej(0), tstart(0), tsamp(0), period(0),
          fch1(0), foff(0), nchans(0), telescope_id(0), machine_id(0), data_type(0), ibeam(0),
          nbeams(0), nbits(0), barycentric(0), pulsarcentric(0), nbins(0), nsamples(0), nifs(0),
          npuls(0), refdm(0), signed_data(0), size(0)
    {
    }

    void from_c(const psx_sigproc_header& h)
    {
        source_name = h.source_name;
        rawdatafile = h.rawdatafile;
        az_start = h.az_start; za_start = h.za_start; src_raj = h.src_raj; src_dej = h.src_dej;
        tstart = h.tstart; tsamp = h.tsamp; period = h.period; fch1 = h.fch1; foff = h.foff;
        nchans = h.nchans; telescope_id = h.telescope_id; machine_id = h.machine_id;
        data_type = h.data_type; ibeam = h.ibeam; nbeams = h.nbeams; nbits = h.nbits;
        barycentric = h.barycentric; pulsarcentric = h.pulsarcentric; nbins = h.nbins;
        nsamples = h.nsamples; nifs = h.nifs; npuls = h.npuls; refdm = h.refdm;
        signed_data = h.signed_data;
        size = (unsigned int)h.header_size;
    }

    psx_sigproc_header to_c() const
    {
        psx_sigproc_header h;
        std::memset(&h, 0, sizeof(h));
        std::strncpy(h.source_name, source_name.c_str(), sizeof(h.source_name) - 1);
        std::strncpy(h.rawdatafile, rawdatafile.c_str(), sizeof(h.rawdatafile) - 1);
        h.az_start = az_start; h.za_start = za_start; h.src_raj = src_raj; h.src_dej = src_dej;
        h.tstart = tstart; h.tsamp = tsamp; h.period = period; h.fch1 = fch1; h.foff = foff;
        h.nchans = nchans; h.telescope_id = telescope_id; h.machine_id = machine_id;
        h.data_type = data_type; h.ibeam = ibeam; h.nbeams = nbeams; h.nbits = nbits;
        h.barycentric = barycentric; h.pulsarcentric = pulsarcentric; h.nbins = nbins;
        h.nsamples = nsamples; h.nifs = nifs; h.npuls = npuls; h.refdm = refdm;
        h.signed_data = signed_data;
        h.header_size = size;
        return h;
    }
};

// Reads the header at the start of `stream` into `header` and leaves the
// stream at the first sample.  nsamples == 0 in the file is replaced by
// (file size - header size) / nchans * 8 / nbits.  Returns false (and
// rewinds the stream) when the stream holds no SIGPROC header; the
// reference returned false in every case and its callers ignore the value.
template <class BinaryStream, class Header>
bool read_header(BinaryStream& stream, Header& header)
{
    stream.clear();
    stream.seekg(0, std::ios::end);
    const size_t total = (size_t)stream.tellg();
    std::vector<char> buf;
    psx_sigproc_header h;
    int rc = PSX_ERR_OVERFLOW;
    for (size_t want = 4096; rc == PSX_ERR_OVERFLOW; want *= 4) {
        size_t k = want < total ? want : total;
        buf.resize(k ? k : 1);
        stream.clear();
        stream.seekg(0, std::ios::beg);
        stream.read(buf.data(), (std::streamsize)k);
        rc = psx_sigproc_parse_header(buf.data(), (size_t)stream.gcount(), &h);
        if (rc == PSX_ERR_OVERFLOW && k == total) break;
    }
    stream.clear();
    if (rc != PSX_OK) {
        stream.seekg(0, std::ios::beg);
        return false;
    }
    if (h.nsamples == 0 && h.nchans > 0 && h.nbits > 0) {
        size_t data = total >= h.header_size ? total - h.header_size : 0;
        h.nsamples = (int)(data / (size_t)h.nchans * 8 / (size_t)h.nbits);
    }
    header.from_c(h);
    stream.seekg((std::streamoff)h.header_size, std::ios::beg);
    return true;
}
