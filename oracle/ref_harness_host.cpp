/*
 * ref_harness_host.cpp -- drives the reference's own host-side classes of
 * the search path that need no GPU: AccelerationPlan
 * (include/utils/utils.hpp:143-233) and the candidate distillers
 * (include/transforms/distiller.hpp).  Compiled with g++ from the reference
 * headers where they lie, into oracle/_ref/; runs on any CPU.
 *
 * TEST INFRASTRUCTURE ONLY: used to pin the oracle and the product's host
 * logic; never linked by the product.
 */
#include <cstring>
#include <vector>
#include <utils/utils.hpp>
#include <data_types/candidates.hpp>
#include <transforms/distiller.hpp>

extern "C" {

typedef struct {
    float dm;
    int dm_idx;
    float acc;
    int nh;
    float snr;
    float freq;
} ref_candidate;

/* AccelerationPlan(...).generate_accel_list(dm, cdm, list). */
size_t ref_accel_list(float acc_lo, float acc_hi, float tol, float pulse_width_s,
                      size_t nsamps, float tsamp, float cfreq_hz, float ch_bw_hz,
                      float dm, float cdm, float* out, size_t cap)
{
    AccelerationPlan plan(acc_lo, acc_hi, tol, pulse_width_s, nsamps, tsamp,
                          cfreq_hz, ch_bw_hz);
    std::vector<float> v;
    plan.generate_accel_list(dm, cdm, v);
    for (size_t i = 0; i < v.size() && i < cap; ++i) out[i] = v[i];
    return v.size();
}

/* kind 0: HarmonicDistiller(tol, max_harm, keep_related, fractional)
   kind 1: AccelerationDistiller(tobs, tol, keep_related)
   kind 2: DMDistiller(tol, keep_related)
   Writes the survivors in the reference's output order and each one's
   Candidate::count_assoc(). */
size_t ref_distill(int kind, const ref_candidate* in, size_t n, float tol, float max_harm,
                   float tobs, int keep_related, int fractional, ref_candidate* out,
                   int* nassoc)
{
    std::vector<Candidate> c;
    c.reserve(n);
    for (size_t i = 0; i < n; ++i)
        c.push_back(Candidate(in[i].dm, in[i].dm_idx, in[i].acc, in[i].nh, in[i].snr, in[i].freq));
    std::vector<Candidate> r;
    if (kind == 0) {
        HarmonicDistiller d(tol, max_harm, keep_related != 0, fractional != 0);
        r = d.distill(c);
    } else if (kind == 1) {
        AccelerationDistiller d(tobs, tol, keep_related != 0);
        r = d.distill(c);
    } else {
        DMDistiller d(tol, keep_related != 0);
        r = d.distill(c);
    }
    for (size_t i = 0; i < r.size(); ++i) {
        out[i] = ref_candidate{r[i].dm, r[i].dm_idx, r[i].acc, r[i].nh, r[i].snr, r[i].freq};
        if (nassoc) nassoc[i] = r[i].count_assoc();
    }
    return r.size();
}

}  // extern "C"
