// scorer.hpp -- CandidateScorer of the drop-in API (reference
// include/transforms/scorer.hpp:8-87), over psx_score_forest: for every
// candidate, from its direct associations, whether its period exceeds the
// channel DM smearing (is_physical), whether an association sits one DM
// trial away or none off its DM trial (is_adjacent), and the shares of
// associations and of their S/N within the DM width of its period
// (ddm_count_ratio, ddm_snr_ratio).  Frequencies in MHz, as the reference
// passes them (src/pipeline_multi.cu:550-552).
#pragma once
#include <stdexcept>
#include <string>
#include <vector>
#include "data_types/candidates.hpp"
#include "peasoup_b200.h"

class CandidateScorer {
    float tsamp, cfreq, foff, bw;

public:
    CandidateScorer(float tsamp_, float cfreq_, float foff_, float bw_)
        : tsamp(tsamp_), cfreq(cfreq_), foff(foff_), bw(bw_)
    {
    }

    void score_all(std::vector<Candidate>& cands)
    {
        if (cands.empty()) return;
        // only the direct associations are scored: a depth-one forest
        std::vector<psx_candidate> nodes;
        std::vector<int> sizes;
        for (const Candidate& c : cands) {
            nodes.push_back(c.pod());
            sizes.push_back(1 + (int)c.assoc.size());
            for (const Candidate& a : c.assoc) {
                nodes.push_back(a.pod());
                sizes.push_back(1);
            }
        }
        std::vector<psx_candidate_score> s(cands.size());
        size_t n = 0;
        const int rc = psx_score_forest(nodes.data(), sizes.data(), nodes.size(), tsamp, cfreq,
                                        foff, bw, s.data(), s.size(), &n);
        if (rc != PSX_OK) throw std::runtime_error(std::string("score: ") + psx_last_error());
        for (size_t i = 0; i < cands.size(); ++i) {
            cands[i].is_physical = s[i].is_physical != 0;
            cands[i].is_adjacent = s[i].is_adjacent != 0;
            cands[i].ddm_count_ratio = s[i].ddm_count_ratio;
            cands[i].ddm_snr_ratio = s[i].ddm_snr_ratio;
        }
    }

    void score(Candidate& cand)
    {
        std::vector<Candidate> one(1, cand);
        score_all(one);
        cand.is_physical = one[0].is_physical;
        cand.is_adjacent = one[0].is_adjacent;
        cand.ddm_count_ratio = one[0].ddm_count_ratio;
        cand.ddm_snr_ratio = one[0].ddm_snr_ratio;
    }
};
