// candidates.hpp -- candidate records of the drop-in API (reference
// include/data_types/candidates.hpp:10-166).  CandidatePOD has the same
// six fields in the same order (the 24-byte record of candidates.peasoup)
// and the same layout as psx_candidate.  A Candidate carries its
// association tree in `assoc`, as the reference's does; to_forest /
// from_forest convert trees to and from the library's candidate forests
// (nodes in depth-first order with subtree sizes).
#pragma once
#include <cstdio>
#include <vector>
#include "peasoup_b200.h"

struct CandidatePOD {
    float dm;
    int dm_idx;
    float acc;
    int nh;
    float snr;
    float freq;
};
static_assert(sizeof(CandidatePOD) == sizeof(psx_candidate), "record layout");

struct Candidate {
    float dm = 0.f;
    int dm_idx = 0;
    float acc = 0.f;
    int nh = 0;
    float snr = 0.f;
    float freq = 0.f;
    float folded_snr = 0.f;
    double opt_period = 0.0;
    bool is_adjacent = false;
    bool is_physical = false;
    float ddm_count_ratio = 0.f;
    float ddm_snr_ratio = 0.f;
    std::vector<Candidate> assoc;
    std::vector<float> fold;
    int nbins = 0;
    int nints = 0;

    Candidate() {}
    Candidate(float dm_, int dm_idx_, float acc_, int nh_, float snr_, float freq_)
        : dm(dm_), dm_idx(dm_idx_), acc(acc_), nh(nh_), snr(snr_), freq(freq_)
    {
    }
    Candidate(float dm_, int dm_idx_, float acc_, int nh_, float snr_, float folded_snr_,
              float freq_)
        : dm(dm_), dm_idx(dm_idx_), acc(acc_), nh(nh_), snr(snr_), freq(freq_),
          folded_snr(folded_snr_)
    {
    }
    explicit Candidate(const psx_candidate& c)
        : dm(c.dm), dm_idx(c.dm_idx), acc(c.acc), nh(c.nh), snr(c.snr), freq(c.freq)
    {
    }
    void append(const Candidate& other) { assoc.push_back(other); }
    int count_assoc() const
    {
        int n = 0;
        for (const Candidate& a : assoc) n += 1 + a.count_assoc();
        return n;
    }
    psx_candidate pod() const { return psx_candidate{dm, dm_idx, acc, nh, snr, freq}; }
    void set_fold(const float* ar, int nbins_, int nints_)
    {
        nbins = nbins_;
        nints = nints_;
        fold.assign(ar, ar + (size_t)nbins_ * nints_);
    }
    // This candidate and its associations, depth first (the records of
    // candidates.peasoup).
    void collect_candidates(std::vector<CandidatePOD>& out) const
    {
        out.push_back(CandidatePOD{dm, dm_idx, acc, nh, snr, freq});
        for (const Candidate& a : assoc) a.collect_candidates(out);
    }
    // Appends the tree to a candidate forest.
    void to_forest(std::vector<psx_candidate>& nodes, std::vector<int>& sizes) const
    {
        const size_t at = nodes.size();
        nodes.push_back(pod());
        sizes.push_back(0);
        for (const Candidate& a : assoc) a.to_forest(nodes, sizes);
        sizes[at] = (int)(nodes.size() - at);
    }
    // The tree rooted at nodes[i]; advances i past it.
    static Candidate from_forest(const psx_candidate* nodes, const int* sizes, size_t& i)
    {
        Candidate c(nodes[i]);
        const size_t end = i + (size_t)sizes[i];
        ++i;
        while (i < end) c.assoc.push_back(from_forest(nodes, sizes, i));
        return c;
    }
    void print(FILE* fo = stdout) const
    {
        std::fprintf(fo, "%.15f\t%.15f\t%.15f\t%.2f\t%.2f\t%d\t%.1f\t%.1f\t%d\t%d\t%.4f\t%.4f\t%zu\n",
                     1.0 / freq, opt_period, (double)freq, (double)dm, (double)acc, nh,
                     (double)snr, (double)folded_snr, (int)is_adjacent, (int)is_physical,
                     (double)ddm_count_ratio, (double)ddm_snr_ratio, assoc.size());
        for (const Candidate& a : assoc) a.print(fo);
    }
};

// A forest from a list of trees, and back.
inline void to_forest(const std::vector<Candidate>& cands, std::vector<psx_candidate>& nodes,
                      std::vector<int>& sizes)
{
    nodes.clear();
    sizes.clear();
    for (const Candidate& c : cands) c.to_forest(nodes, sizes);
}

inline std::vector<Candidate> from_forest(const psx_candidate* nodes, const int* sizes, size_t n)
{
    std::vector<Candidate> out;
    size_t i = 0;
    while (i < n) out.push_back(Candidate::from_forest(nodes, sizes, i));
    return out;
}

class CandidateCollection {
public:
    std::vector<Candidate> cands;
    void append(const CandidateCollection& o) { cands.insert(cands.end(), o.cands.begin(), o.cands.end()); }
    void append(const std::vector<Candidate>& o) { cands.insert(cands.end(), o.begin(), o.end()); }
    void reset() { cands.clear(); }
    void print(FILE* fo = stdout) const
    {
        for (const Candidate& c : cands) c.print(fo);
    }
};

class SpectrumCandidates : public CandidateCollection {
public:
    float dm;
    int dm_idx;
    float acc;
    SpectrumCandidates(float dm_, int dm_idx_, float acc_) : dm(dm_), dm_idx(dm_idx_), acc(acc_) {}
    void append(const float* snrs, const float* freqs, int nh, int size)
    {
        for (int i = 0; i < size; ++i) cands.push_back(Candidate(dm, dm_idx, acc, nh, snrs[i], freqs[i]));
    }
};
