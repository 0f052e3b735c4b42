// distiller.hpp -- candidate distillers of the drop-in API (reference
// include/transforms/distiller.hpp:16-196).  distill() sorts the input by
// descending S/N in place, as the reference does, and returns the
// survivors; with keep_related each survivor carries its association tree
// in `assoc` (the absorbed candidates with their own trees, in the
// reference's append order), computed by psx_distill_forest.
#pragma once
#include <algorithm>
#include <stdexcept>
#include <string>
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
        std::vector<psx_candidate> nodes, out;
        std::vector<int> sizes, out_sizes;
        to_forest(cands, nodes, sizes);
        size_t n = 0;
        int rc = psx_distill_forest(kind, nodes.data(), sizes.data(), nodes.size(), tol, max_harm,
                                    tobs, keep_related, fractional, nullptr, nullptr, 0, &n,
                                    nullptr);
        if (rc == PSX_ERR_OVERFLOW || rc == PSX_OK) {
            out.resize(n);
            out_sizes.resize(n);
            rc = psx_distill_forest(kind, nodes.data(), sizes.data(), nodes.size(), tol, max_harm,
                                    tobs, keep_related, fractional, out.data(), out_sizes.data(),
                                    n, &n, nullptr);
        }
        if (rc != PSX_OK) throw std::runtime_error(std::string("distill: ") + psx_last_error());
        // the reference sorts its input by descending S/N in place
        std::sort(cands.begin(), cands.end(),
                  [](const Candidate& a, const Candidate& b) { return a.snr > b.snr; });
        return from_forest(out.data(), out_sizes.data(), n);
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
