// dropin_dedisp.cpp -- the reference main program's input side
// (src/pipeline_multi.cu:378-505) written against the drop-in headers:
// SigprocFilterbank, read_header, Dedisperser (generate_dm_list or a DM
// file, optional killfile), DispersionTrials.  Writes the header values it
// read, the DM list and the dedispersed block to a binary file:
//   int32 ndm, int64 nsamps, int64 header size, int32 nchans, int32 nbits,
//   float32 tsamp, fch1, foff, cfreq; float32 dms[ndm];
//   float32 data[ndm][nsamps].
//
//   dropin_dedisp <fil> <start> <nsamples> <dm_start> <dm_end> <out> [dm_file|-] [killfile]
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include "data_types/filterbank.hpp"
#include "data_types/header.hpp"
#include "data_types/timeseries.hpp"
#include "transforms/dedisperser.hpp"

int main(int argc, char** argv)
{
    if (argc < 7) {
        std::fprintf(stderr, "usage: %s fil start nsamples dm_start dm_end out [dm_file|-] [killfile]\n",
                     argv[0]);
        return 2;
    }
    try {
        std::string fil = argv[1];
        SigprocFilterbank filobj(fil, std::strtoull(argv[2], nullptr, 10),
                                 std::strtoull(argv[3], nullptr, 10));
        // the stream form the reference's output writer uses
        std::ifstream in(fil.c_str(), std::ifstream::in | std::ifstream::binary);
        SigprocHeader hdr;
        read_header(in, hdr);
        if (hdr.size != filobj.get_header().size || hdr.nsamples != filobj.get_header().nsamples ||
            hdr.source_name != filobj.get_header().source_name) {
            std::fprintf(stderr, "stream and path headers differ\n");
            return 3;
        }
        Dedisperser dd(filobj, 1);
        if (argc > 7 && std::string(argv[7]) != "-") {
            std::vector<float> dms;
            std::ifstream f(argv[7]);
            std::string line;
            float v = 0;
            while (std::getline(f, line)) {
                if (!line.empty()) v = (float)std::atof(line.c_str());
                dms.push_back(v);
            }
            dd.set_dm_list(dms);
        } else {
            dd.generate_dm_list((float)std::atof(argv[4]), (float)std::atof(argv[5]), 64.0f, 1.11f);
        }
        if (argc > 8) dd.set_killmask(std::string(argv[8]));
        DispersionTrials<float> trials(filobj.get_tsamp());
        dd.dedisperse(trials, filobj.get_start_sample(), filobj.get_end_sample(), 4096);
        std::vector<float> dms = dd.get_dm_list();
        FILE* out = std::fopen(argv[6], "wb");
        if (!out) return 4;
        int ndm = (int)dms.size();
        long long ns = (long long)trials.get_nsamps(), hs = hdr.size;
        int nch = hdr.nchans, nb = hdr.nbits;
        float meta[4] = {filobj.get_tsamp(), filobj.get_fch1(), filobj.get_foff(),
                         filobj.get_cfreq()};
        std::fwrite(&ndm, 4, 1, out);
        std::fwrite(&ns, 8, 1, out);
        std::fwrite(&hs, 8, 1, out);
        std::fwrite(&nch, 4, 1, out);
        std::fwrite(&nb, 4, 1, out);
        std::fwrite(meta, 4, 4, out);
        std::fwrite(dms.data(), 4, dms.size(), out);
        std::fwrite(trials.get_data_ptr(), 4, (size_t)ndm * (size_t)ns, out);
        std::fclose(out);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
