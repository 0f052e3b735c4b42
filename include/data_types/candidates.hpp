// candidates.hpp -- candidate records of the drop-in API (reference
// include/data_types/candidates.hpp:10-166).  CandidatePOD has the same
// six fields in the same order (the 24-byte record of candidates.peasoup)
// and the same layout as psx_candidate.
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
    std::vector<Candidate> assoc;

    Candidate() {}
    Candidate(float dm_, int dm_idx_, float acc_, int nh_, float snr_, float freq_)
        : dm(dm_), dm_idx(dm_idx_), acc(acc_), nh(nh_), snr(snr_), freq(freq_)
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
};

class CandidateCollection {
public:
    std::vector<Candidate> cands;
    void append(const CandidateCollection& o) { cands.insert(cands.end(), o.cands.begin(), o.cands.end()); }
    void append(const std::vector<Candidate>& o) { cands.insert(cands.end(), o.begin(), o.end()); }
    void reset() { cands.clear(); }
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
