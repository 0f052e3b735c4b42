/*
 * ref_harness_host.cpp -- drives the reference's own host-side classes of
 * the search path that need no GPU: AccelerationPlan
 * (include/utils/utils.hpp:143-233), the candidate distillers
 * (include/transforms/distiller.hpp), CandidateScorer
 * (include/transforms/scorer.hpp) and the output writers
 * (include/utils/output_stats.hpp).  Candidate trees cross this boundary as
 * forests: nodes in depth-first order with subtree sizes.  Compiled with g++ from the reference
 * headers where they lie, into oracle/_ref/; runs on any CPU.
 *
 * TEST INFRASTRUCTURE ONLY: used to pin the oracle and the product's host
 * logic; never linked by the product.
 */
#include <cuda_runtime.h>
#include <cstring>
#include <string>
#include <vector>
#include <utils/utils.hpp>
#include <utils/exceptions.hpp>
#include <data_types/candidates.hpp>
#include <data_types/filterbank.hpp>
#include <transforms/distiller.hpp>
#include <transforms/scorer.hpp>
#include <utils/output_stats.hpp>

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

/* ---- candidate forests <-> Candidate trees ---- */
static Candidate tree_at(const ref_candidate* nodes, const int* sizes, size_t& i)
{
    Candidate c(nodes[i].dm, nodes[i].dm_idx, nodes[i].acc, nodes[i].nh, nodes[i].snr,
                nodes[i].freq);
    const size_t end = i + (size_t)sizes[i];
    ++i;
    while (i < end) {
        Candidate child = tree_at(nodes, sizes, i);
        c.append(child);
    }
    return c;
}

static std::vector<Candidate> trees(const ref_candidate* nodes, const int* sizes, size_t n)
{
    std::vector<Candidate> out;
    size_t i = 0;
    while (i < n) out.push_back(tree_at(nodes, sizes, i));
    return out;
}

static void flatten(Candidate& c, std::vector<ref_candidate>& out, std::vector<int>& sizes)
{
    const size_t at = out.size();
    out.push_back(ref_candidate{c.dm, c.dm_idx, c.acc, c.nh, c.snr, c.freq});
    sizes.push_back(0);
    for (size_t k = 0; k < c.assoc.size(); ++k) flatten(c.assoc[k], out, sizes);
    sizes[at] = (int)(out.size() - at);
}

/* The distillers on trees; writes the survivors' trees as a forest and
   returns its node count (or the need when larger than cap). */
size_t ref_distill_forest(int kind, const ref_candidate* nodes, const int* sizes, size_t n,
                          float tol, float max_harm, float tobs, int keep_related,
                          int fractional, ref_candidate* out, int* out_sizes, size_t cap)
{
    std::vector<Candidate> c = trees(nodes, sizes, n);
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
    std::vector<ref_candidate> f;
    std::vector<int> fs;
    for (size_t i = 0; i < r.size(); ++i) flatten(r[i], f, fs);
    if (f.size() <= cap) {
        std::memcpy(out, f.data(), sizeof(ref_candidate) * f.size());
        std::memcpy(out_sizes, fs.data(), sizeof(int) * fs.size());
    }
    return f.size();
}

typedef struct {
    int is_physical, is_adjacent;
    float ddm_count_ratio, ddm_snr_ratio;
    int nassoc;
} ref_score;

static void score(std::vector<Candidate>& c, float tsamp, float cfreq, float foff, float bw)
{
    CandidateScorer sc(tsamp, cfreq, foff, bw);
    sc.score_all(c);
}

/* CandidateScorer::score_all on the forest's roots. */
size_t ref_score_forest(const ref_candidate* nodes, const int* sizes, size_t n, float tsamp,
                        float cfreq, float foff, float bw, ref_score* out)
{
    std::vector<Candidate> c = trees(nodes, sizes, n);
    score(c, tsamp, cfreq, foff, bw);
    for (size_t i = 0; i < c.size(); ++i)
        out[i] = ref_score{c[i].is_physical ? 1 : 0, c[i].is_adjacent ? 1 : 0,
                           c[i].ddm_count_ratio, c[i].ddm_snr_ratio, c[i].count_assoc()};
    return c.size();
}

/* CandidateFileWriter(dir).write_binary(trees, filename); byte offsets of
   every root. */
size_t ref_write_binary(const char* dir, const char* filename, const ref_candidate* nodes,
                        const int* sizes, size_t n, long long* offsets)
{
    std::vector<Candidate> c = trees(nodes, sizes, n);
    CandidateFileWriter w(dir);
    w.write_binary(c, filename);
    for (size_t i = 0; i < c.size(); ++i) offsets[i] = w.byte_mapping[(unsigned)i];
    return c.size();
}

/* OutputFileWriter with the DM list, the acceleration list and the scored
   candidates (byte offsets given), as text; returns its length. */
size_t ref_overview_text(const float* dms, size_t ndm, const float* accs, size_t nacc, float cdm,
                         const ref_candidate* nodes, const int* sizes, size_t n,
                         const long long* offsets, float tsamp, float cfreq, float foff,
                         float bw, char* out, size_t cap)
{
    std::vector<Candidate> c = trees(nodes, sizes, n);
    score(c, tsamp, cfreq, foff, bw);
    OutputFileWriter w;
    std::vector<float> d(dms, dms + ndm), a(accs, accs + nacc);
    w.add_dm_list(d);
    w.add_acc_list(a, cdm);
    std::map<unsigned, long int> bm;
    for (size_t i = 0; i < c.size(); ++i) bm[(unsigned)i] = (long int)offsets[i];
    w.add_candidates(c, bm);
    const std::string t = w.to_string();
    if (t.size() + 1 <= cap) std::memcpy(out, t.c_str(), t.size() + 1);
    return t.size();
}

}  // extern "C"

/* The reference's SIGPROC reader: read_header (include/data_types/header.hpp:
   339-403) into SigprocHeader, flattened into doubles in a fixed order:
   az_start za_start src_raj src_dej tstart tsamp period fch1 foff refdm
   nchans telescope_id machine_id data_type ibeam nbeams nbits barycentric
   pulsarcentric nbins nsamples nifs npuls signed size (25 values). */
extern "C" int ref_sigproc_header(const char* path, double* out, char* source_name,
                                  char* rawdatafile)
{
    std::ifstream f(path, std::ifstream::in | std::ifstream::binary);
    if (!f) return 1;
    SigprocHeader h;
    read_header(f, h);
    double v[25] = {h.az_start, h.za_start, h.src_raj, h.src_dej, h.tstart, h.tsamp, h.period,
                    h.fch1, h.foff, h.refdm, (double)h.nchans, (double)h.telescope_id,
                    (double)h.machine_id, (double)h.data_type, (double)h.ibeam,
                    (double)h.nbeams, (double)h.nbits, (double)h.barycentric,
                    (double)h.pulsarcentric, (double)h.nbins, (double)h.nsamples,
                    (double)h.nifs, (double)h.npuls, (double)h.signed_data, (double)h.size};
    std::memcpy(out, v, sizeof(v));
    std::snprintf(source_name, 80, "%s", h.source_name.c_str());
    std::snprintf(rawdatafile, 80, "%s", h.rawdatafile.c_str());
    return 0;
}

/* SigprocFilterbank(path, seg_start, seg_n) and one load_gulp(start, n)
   (include/data_types/filterbank.hpp:261-328): the metadata the program
   uses (tsamp, fch1, foff, cfreq as float; start, end, effective) and the
   bytes read. */
extern "C" size_t ref_filterbank_gulp(const char* path, size_t seg_start, size_t seg_n,
                                      size_t start, size_t n, unsigned char* out, size_t cap,
                                      double* meta)
{
    SigprocFilterbank fil(path, seg_start, seg_n);
    size_t got = fil.load_gulp(start, n);
    size_t bytes = got * (size_t)fil.get_nchans() * (size_t)fil.get_nbits() / 8;
    std::memcpy(out, fil.get_data(), std::min(bytes, cap));
    meta[0] = fil.get_tsamp();
    meta[1] = fil.get_fch1();
    meta[2] = fil.get_foff();
    meta[3] = fil.get_cfreq();
    meta[4] = (double)fil.get_start_sample();
    meta[5] = (double)fil.get_end_sample();
    meta[6] = (double)fil.get_effective_nsamps();
    meta[7] = (double)fil.get_total_nsamps();
    fil.size = 1u << 16;
    meta[8] = fil.get_segment_pepoch();
    return got;
}
