// distiller.hpp -- candidate distillers of the drop-in API (reference
// include/transforms/distiller.hpp:16-196).  distill() sorts the input by
// descending S/N in place, as the reference does, and returns the
// survivors; with keep_related each survivor carries its association
// count in `assoc` (as placeholder entries).
#pragma once
#include <vector>
#include "data_types/candidates.hpp"
#include "peasoup_b200.h"

class BaseDistiller {
protected:
    int kind;
    float tol, max_harm, tobs;
    bool keep_related, fractional;
    BaseDistiller(int k, float t, float mh, float to, bool kr, bool fr)
        : kind(k), tol(t), max_harm(mh), tobs(to), keep_related(kr), fractional(fr)
    {
    }

public:
    virtual ~BaseDistiller() {}
    std::vector<Candidate> distill(std::vector<Candidate>& cands)
    {
        std::vector<psx_candidate> pod(cands.size());
        for (size_t i = 0; i < cands.size(); ++i) pod[i] = cands[i].pod();
        std::vector<int> na(cands.size());
        const size_t keep = pod.empty() ? 0
                                        : psx_distill(kind, pod.data(), pod.size(), tol, max_harm,
                                                      tobs, keep_related, fractional, na.data());
        std::vector<Candidate> out;
        out.reserve(keep);
        for (size_t i = 0; i < keep; ++i) {
            Candidate c(pod[i]);
            c.assoc.resize((size_t)na[i]);
            out.push_back(c);
        }
        return out;
    }
};

class HarmonicDistiller : public BaseDistiller {
public:
    HarmonicDistiller(float tol_, float max_harm_, bool keep_related_, bool fractional_harms = true)
        : BaseDistiller(PSX_DISTILL_HARMONIC, tol_, max_harm_, 0.f, keep_related_, fractional_harms)
    {
    }
};

class AccelerationDistiller : public BaseDistiller {
public:
    AccelerationDistiller(float tobs_, float tolerance, bool keep_related_)
        : BaseDistiller(PSX_DISTILL_ACCEL, tolerance, 16.f, tobs_, keep_related_, true)
    {
    }
};

class DMDistiller : public BaseDistiller {
public:
    DMDistiller(float tolerance, bool keep_related_)
        : BaseDistiller(PSX_DISTILL_DM, tolerance, 16.f, 0.f, keep_related_, true)
    {
    }
};
