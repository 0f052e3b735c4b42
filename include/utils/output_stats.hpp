// output_stats.hpp -- the output files of the drop-in API (reference
// include/utils/output_stats.hpp): CandidateFileWriter writes
// candidates.peasoup (psx_write_candidates) and OutputFileWriter builds
// overview.xml (psx_overview_*) in the reference's XML layout.  Sections
// whose values come from outside the search path (the SIGPROC header, the
// command line, the segment) are added with add_section as name/value
// pairs; to_text() formats a number as the reference's writer prints it.
// Candidate folds are not part of this library: no FOLD blocks are written.
#pragma once
#include <cstdio>
#include <ctime>
#include <map>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <utility>
#include <vector>
#include <cuda_runtime.h>
#include "data_types/candidates.hpp"
#include "peasoup_b200.h"

namespace psx_output_detail {
inline void check(int rc, const char* where)
{
    if (rc != PSX_OK) throw std::runtime_error(std::string(where) + ": " + psx_last_error());
}
}  // namespace psx_output_detail

class CandidateFileWriter {
public:
    std::map<unsigned, long int> byte_mapping;
    std::string output_dir;

    explicit CandidateFileWriter(std::string output_directory) : output_dir(std::move(output_directory))
    {
        struct stat st = {};
        if (stat(output_dir.c_str(), &st) == -1 && mkdir(output_dir.c_str(), 0777) != 0)
            std::perror(output_dir.c_str());
    }

    void write_binary(std::vector<Candidate>& candidates, std::string filename)
    {
        std::vector<psx_candidate> nodes;
        std::vector<int> sizes;
        to_forest(candidates, nodes, sizes);
        std::vector<long long> off(candidates.size());
        size_t n = 0;
        const std::string path = output_dir + "/" + filename;
        psx_output_detail::check(psx_write_candidates(path.c_str(), nodes.data(), sizes.data(),
                                                      nodes.size(), off.data(), off.size(), &n),
                                 "write_binary");
        for (size_t i = 0; i < n; ++i) byte_mapping[(unsigned)i] = (long int)off[i];
    }
};

class OutputFileWriter {
    psx_overview* o = nullptr;

public:
    OutputFileWriter() { psx_output_detail::check(psx_overview_create(&o), "overview"); }
    ~OutputFileWriter() { psx_overview_destroy(o); }
    OutputFileWriter(const OutputFileWriter&) = delete;
    OutputFileWriter& operator=(const OutputFileWriter&) = delete;

    static std::string to_text(double v)
    {
        char b[64];
        std::snprintf(b, sizeof b, "%.15g", v);
        return b;
    }
    static std::string to_text(long long v) { return std::to_string(v); }

    void add_section(const std::string& name,
                     const std::vector<std::pair<std::string, std::string>>& items)
    {
        std::vector<const char*> k, v;
        for (const auto& it : items) {
            k.push_back(it.first.c_str());
            v.push_back(it.second.c_str());
        }
        psx_output_detail::check(
            psx_overview_add_section(o, name.c_str(), k.data(), v.data(), items.size()),
            "add_section");
    }
    void add_misc_info()
    {
        psx_output_detail::check(psx_overview_add_misc_info(o, (long long)std::time(nullptr)),
                                 "add_misc_info");
    }
    void add_dm_list(std::vector<float>& dms)
    {
        psx_output_detail::check(psx_overview_add_dm_list(o, dms.data(), dms.size()),
                                 "add_dm_list");
    }
    void add_acc_list(std::vector<float>& accs, float cdm)
    {
        psx_output_detail::check(psx_overview_add_acc_list(o, accs.data(), accs.size(), cdm),
                                 "add_acc_list");
    }
    void add_gpu_info(std::vector<int>& device_idxs)
    {
        int rt = 0, dv = 0;
        cudaRuntimeGetVersion(&rt);
        cudaDriverGetVersion(&dv);
        std::vector<std::string> names;
        std::vector<const char*> np;
        std::vector<int> major, minor;
        for (int d : device_idxs) {
            cudaDeviceProp p{};
            cudaGetDeviceProperties(&p, d);
            names.push_back(p.name);
            major.push_back(p.major);
            minor.push_back(p.minor);
        }
        for (const std::string& s : names) np.push_back(s.c_str());
        psx_output_detail::check(
            psx_overview_add_device_info(o, rt, dv, device_idxs.data(), np.data(), major.data(),
                                         minor.data(), device_idxs.size()),
            "add_gpu_info");
    }
    void add_timing_info(const std::map<std::string, double>& seconds)
    {
        std::vector<std::pair<std::string, std::string>> items;
        for (const auto& it : seconds) items.emplace_back(it.first, to_text(it.second));
        add_section("execution_times", items);
    }
    // Candidates scored by CandidateScorer; byte offsets from
    // CandidateFileWriter::byte_mapping.
    void add_candidates(std::vector<Candidate>& candidates, std::map<unsigned, long int> byte_map)
    {
        std::vector<psx_candidate> nodes;
        std::vector<int> sizes;
        to_forest(candidates, nodes, sizes);
        std::vector<psx_candidate_score> sc(candidates.size());
        std::vector<long long> off(candidates.size());
        for (size_t i = 0; i < candidates.size(); ++i) {
            sc[i].is_physical = candidates[i].is_physical;
            sc[i].is_adjacent = candidates[i].is_adjacent;
            sc[i].ddm_count_ratio = candidates[i].ddm_count_ratio;
            sc[i].ddm_snr_ratio = candidates[i].ddm_snr_ratio;
            sc[i].nassoc = candidates[i].count_assoc();
            off[i] = byte_map[(unsigned)i];
        }
        psx_output_detail::check(psx_overview_add_candidates(o, nodes.data(), sizes.data(),
                                                             nodes.size(), sc.data(), off.data()),
                                 "add_candidates");
    }
    std::string to_string()
    {
        size_t n = 0;
        psx_output_detail::check(psx_overview_write(o, nullptr, nullptr, 0, &n), "to_string");
        std::string s(n + 1, '\0');
        psx_output_detail::check(psx_overview_write(o, nullptr, &s[0], s.size(), &n), "to_string");
        s.resize(n);
        return s;
    }
    void to_file(std::string filename)
    {
        size_t n = 0;
        psx_output_detail::check(psx_overview_write(o, filename.c_str(), nullptr, 0, &n),
                                 "to_file");
    }
};
