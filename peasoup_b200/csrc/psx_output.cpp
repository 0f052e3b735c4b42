// psx_output.cpp -- what the reference does with the candidates after its
// Workers: distillation of candidate trees across DM trials and harmonics
// (include/transforms/distiller.hpp:16-196 with keep_related), scoring
// (include/transforms/scorer.hpp:8-87), and the two output files
// candidates.peasoup and overview.xml (include/utils/output_stats.hpp).
//
// A candidate forest is a node array in depth-first order plus, per node,
// the size of the subtree it roots (itself included).  It is the
// reference's Candidate::assoc tree laid out the way
// Candidate::collect_candidates walks it (candidates.hpp:80-86), so a root's
// subtree is exactly the run of records candidates.peasoup holds for it.
// Roots are the nodes that start a top-level subtree.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <string>
#include <vector>
#include "peasoup_b200.h"
#include "psx_host.h"

namespace psx {
void set_error(const char* fmt, ...);
void clear_error();
}  // namespace psx

namespace {

// Start index of every top-level subtree; false if the sizes do not tile
// the array (a child running past its parent's end, or a size < 1).
bool forest_roots(const int* sizes, size_t n, std::vector<size_t>* roots)
{
    roots->clear();
    // every subtree's children must tile it exactly: check with an explicit
    // stack of open subtree ends
    std::vector<size_t> ends;
    for (size_t i = 0; i < n; ++i) {
        while (!ends.empty() && ends.back() == i) ends.pop_back();
        if (sizes[i] < 1) return false;
        const size_t end = i + (size_t)sizes[i];
        if (end > n) return false;
        if (!ends.empty() && end > ends.back()) return false;
        if (ends.empty()) roots->push_back(i);
        ends.push_back(end);
    }
    return true;
}

// Direct children of the subtree rooted at r.
void children_of(const int* sizes, size_t r, std::vector<size_t>* out)
{
    out->clear();
    const size_t end = r + (size_t)sizes[r];
    for (size_t c = r + 1; c < end; c += (size_t)sizes[c]) out->push_back(c);
}

struct SnrGreaterIdx {
    const psx_candidate* c;
    bool operator()(size_t a, size_t b) const { return c[a].snr > c[b].snr; }
};

// Number of times the reference's condition() appends candidate b to a
// (0: unrelated).  Harmonic: one append per matching (j, k) ratio pair,
// distiller.hpp:82-90; acceleration: distiller.hpp:126-140; DM: :168-174.
int relation(int kind, const psx_candidate& a, const psx_candidate& b, float tol, float max_harm,
             double tobs_over_c, int fractional)
{
    const double fundi = a.freq;
    // `1 + tolerance` is a float sum there (distiller.hpp:76-77, 164-165)
    const double upper = (double)(1.0f + tol), lower = (double)(1.0f - tol);
    if (kind == PSX_DISTILL_HARMONIC) {
        const float maxden = fractional ? (float)std::pow(2.0, b.nh) : 1.0f;
        const double freq = b.freq;
        int m = 0;
        for (int j = 1; j <= max_harm; ++j)
            for (int k = 1; k <= maxden; ++k) {
                const double ratio = k * freq / (j * fundi);
                if (ratio > lower && ratio < upper) ++m;
            }
        return m;
    }
    if (kind == PSX_DISTILL_ACCEL) {
        const double edge = fundi * tol;
        const double dacc = (double)a.acc - b.acc;
        const double acc_freq = (float)(fundi + dacc * fundi * tobs_over_c);
        if (acc_freq > fundi) return (b.freq > fundi - edge && b.freq < acc_freq + edge) ? 1 : 0;
        return (b.freq < fundi + edge && b.freq > acc_freq - edge) ? 1 : 0;
    }
    const double ratio = b.freq / fundi;
    return (ratio > lower && ratio < upper) ? 1 : 0;
}

// ------------------------------------------------------------------ XML
// An element of overview.xml, written as the reference's XML::Element
// writes it (include/utils/xml_util.hpp): attributes sorted by name and
// single-quoted, two spaces of indent per level, text inline when there are
// no children.
struct Xml {
    std::string name, text;
    std::map<std::string, std::string> attrs;
    std::vector<Xml> kids;
    explicit Xml(std::string n, std::string t = "") : name(std::move(n)), text(std::move(t)) {}
    void write(std::string& out, int level) const
    {
        out.append(2 * (size_t)level, ' ');
        out += "<" + name;
        for (const auto& a : attrs) out += " " + a.first + "='" + a.second + "'";
        out += ">";
        if (kids.empty()) {
            out += text;
        } else {
            out += "\n";
            for (const Xml& k : kids) k.write(out, level + 1);
            out.append(2 * (size_t)level, ' ');
        }
        out += "</" + name + ">\n";
    }
};

// Numbers as a stream with precision 15 prints them (the reference's
// set_text / add_attribute): %.15g of the value (a float widened exactly).
std::string num(double v)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.15g", v);
    return b;
}
std::string num(long long v) { return std::to_string(v); }
std::string fixed4(double v)
{
    char b[64];
    std::snprintf(b, sizeof b, "%.4f", v);
    return b;
}

}  // namespace

struct psx_overview {
    Xml root{"peasoup_search"};
};

extern "C" {

int psx_distill_forest(int kind, const psx_candidate* nodes, const int* sizes, size_t n_nodes,
                       float tol, float max_harm, float tobs, int keep_related, int fractional,
                       psx_candidate* h_out, int* h_out_sizes, size_t cap, size_t* n_out,
                       size_t* n_roots)
{
    psx::clear_error();
    if (!n_out || (n_nodes && (!nodes || !sizes)) || kind < PSX_DISTILL_HARMONIC ||
        kind > PSX_DISTILL_DM) {
        psx::set_error("distill_forest: bad arguments");
        return PSX_ERR_INVALID;
    }
    *n_out = 0;
    if (n_roots) *n_roots = 0;
    std::vector<size_t> roots;
    if (!forest_roots(sizes, n_nodes, &roots)) {
        psx::set_error("distill_forest: subtree sizes do not describe a forest");
        return PSX_ERR_INVALID;
    }
    // BaseDistiller::distill (distiller.hpp:25-57): sort by S/N (the same
    // std::sort, so ties land as the reference's land), then each remaining
    // unique candidate in turn absorbs every later related one
    std::vector<size_t> ord = roots;
    std::sort(ord.begin(), ord.end(), SnrGreaterIdx{nodes});
    const size_t n = ord.size();
    const double tobs_over_c = (double)tobs / 299792458.0;
    std::vector<char> uniq(n, 1);
    std::vector<std::vector<size_t>> app(n);
    for (size_t i = 0; i < n; ++i) {
        if (!uniq[i]) continue;
        const psx_candidate& a = nodes[ord[i]];
        for (size_t j = i + 1; j < n; ++j) {
            const int m = relation(kind, a, nodes[ord[j]], tol, max_harm, tobs_over_c, fractional);
            if (!m) continue;
            uniq[j] = 0;
            if (keep_related)
                for (int r = 0; r < m; ++r) app[i].push_back(ord[j]);
        }
    }
    // survivors in sorted order, each followed by its own subtree and then
    // the subtrees appended to it
    size_t need = 0, nr = 0;
    for (size_t i = 0; i < n; ++i) {
        if (!uniq[i]) continue;
        ++nr;
        need += (size_t)sizes[ord[i]];
        for (size_t b : app[i]) need += (size_t)sizes[b];
    }
    *n_out = need;
    if (n_roots) *n_roots = nr;
    if (need > cap || (need && (!h_out || !h_out_sizes))) {
        psx::set_error("distill_forest: %zu nodes, buffer holds %zu", need, cap);
        return PSX_ERR_OVERFLOW;
    }
    size_t k = 0;
    for (size_t i = 0; i < n; ++i) {
        if (!uniq[i]) continue;
        const size_t r = ord[i], root_at = k;
        std::memcpy(h_out + k, nodes + r, sizeof(psx_candidate) * (size_t)sizes[r]);
        std::memcpy(h_out_sizes + k, sizes + r, sizeof(int) * (size_t)sizes[r]);
        k += (size_t)sizes[r];
        for (size_t b : app[i]) {
            std::memcpy(h_out + k, nodes + b, sizeof(psx_candidate) * (size_t)sizes[b]);
            std::memcpy(h_out_sizes + k, sizes + b, sizeof(int) * (size_t)sizes[b]);
            k += (size_t)sizes[b];
        }
        h_out_sizes[root_at] = (int)(k - root_at);
    }
    return PSX_OK;
}

int psx_score_forest(const psx_candidate* nodes, const int* sizes, size_t n_nodes, float tsamp,
                     float cfreq, float foff, float bw, psx_candidate_score* h_scores,
                     size_t cap, size_t* n_roots)
{
    psx::clear_error();
    (void)tsamp;  // kept by the reference's scorer but not used in its scores
    if (!n_roots || (n_nodes && (!nodes || !sizes))) {
        psx::set_error("score_forest: bad arguments");
        return PSX_ERR_INVALID;
    }
    std::vector<size_t> roots, kids;
    if (!forest_roots(sizes, n_nodes, &roots)) {
        psx::set_error("score_forest: subtree sizes do not describe a forest");
        return PSX_ERR_INVALID;
    }
    *n_roots = roots.size();
    if (roots.size() > cap || (!roots.empty() && !h_scores)) {
        psx::set_error("score_forest: %zu roots, buffer holds %zu", roots.size(), cap);
        return PSX_ERR_OVERFLOW;
    }
    // CandidateScorer's constants (scorer.hpp:64-71), float as there
    const float ftop = (float)((double)cfreq + (double)bw / 2.0);
    const float fbottom = (float)((double)cfreq - (double)bw / 2.0);
    const float tdm_chan_partial = (float)(8300.0 * (double)foff / std::pow((double)cfreq, 3.0));
    const float tdm_band_partial =
        (float)(4150.0 * (1.0 / std::pow((double)fbottom, 2) - 1.0 / std::pow((double)ftop, 2)));
    for (size_t q = 0; q < roots.size(); ++q) {
        const psx_candidate& c = nodes[roots[q]];
        children_of(sizes, roots[q], &kids);
        psx_candidate_score s{};
        // has_physical_period (scorer.hpp:25-27)
        const float tdm_chan = c.dm * tdm_chan_partial;
        s.is_physical = (1.0 / (double)c.freq > (double)tdm_chan) ? 1 : 0;
        // has_adjacency (scorer.hpp:29-44): adjacent if a direct association
        // is one DM trial away, else unique if all share this DM trial
        bool adjacent = false, unique = true;
        for (size_t k : kids) {
            if (nodes[k].dm_idx != c.dm_idx) unique = false;
            if (nodes[k].dm_idx == c.dm_idx + 1 || nodes[k].dm_idx == c.dm_idx - 1) {
                adjacent = true;
                break;
            }
        }
        s.is_adjacent = (adjacent || unique) ? 1 : 0;
        // delta_dm_ratio (scorer.hpp:46-62)
        int inside = 1, total = 1;
        float inside_snr = c.snr, total_snr = c.snr;
        const float ddm = (float)(1.0 / (double)(c.freq * tdm_band_partial));
        for (size_t k : kids) {
            ++total;
            total_snr += nodes[k].snr;
            if (std::fabs(c.dm - nodes[k].dm) <= ddm) {
                ++inside;
                inside_snr += nodes[k].snr;
            }
        }
        s.ddm_count_ratio = (float)inside / (float)total;
        s.ddm_snr_ratio = inside_snr / total_snr;
        s.nassoc = sizes[roots[q]] - 1;
        h_scores[q] = s;
    }
    return PSX_OK;
}

int psx_write_candidates(const char* path, const psx_candidate* nodes, const int* sizes,
                         size_t n_nodes, long long* h_offsets, size_t cap, size_t* n_roots)
{
    psx::clear_error();
    if (!path || !n_roots || (n_nodes && (!nodes || !sizes))) {
        psx::set_error("write_candidates: bad arguments");
        return PSX_ERR_INVALID;
    }
    std::vector<size_t> roots;
    if (!forest_roots(sizes, n_nodes, &roots)) {
        psx::set_error("write_candidates: subtree sizes do not describe a forest");
        return PSX_ERR_INVALID;
    }
    *n_roots = roots.size();
    if (h_offsets && roots.size() > cap) {
        psx::set_error("write_candidates: %zu roots, offset buffer holds %zu", roots.size(), cap);
        return PSX_ERR_OVERFLOW;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        psx::set_error("write_candidates: cannot open %s", path);
        return PSX_ERR_IO;
    }
    // CandidateFileWriter::write_binary (output_stats.hpp:270-298) without
    // folds: per candidate an int record count, then its subtree's records
    long long off = 0;
    bool ok = true;
    for (size_t q = 0; q < roots.size() && ok; ++q) {
        if (h_offsets) h_offsets[q] = off;
        const int nd = sizes[roots[q]];
        ok = std::fwrite(&nd, sizeof(int), 1, f) == 1 &&
             std::fwrite(nodes + roots[q], sizeof(psx_candidate), (size_t)nd, f) == (size_t)nd;
        off += (long long)sizeof(int) + (long long)sizeof(psx_candidate) * nd;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        psx::set_error("write_candidates: write to %s failed", path);
        return PSX_ERR_IO;
    }
    return PSX_OK;
}

// ------------------------------------------------------------ overview.xml
int psx_overview_create(psx_overview** out)
{
    if (!out) return PSX_ERR_INVALID;
    *out = new (std::nothrow) psx_overview;
    return *out ? PSX_OK : PSX_ERR_ALLOC;
}

void psx_overview_destroy(psx_overview* o) { delete o; }

int psx_overview_add_section(psx_overview* o, const char* section, const char* const* keys,
                             const char* const* values, size_t n)
{
    psx::clear_error();
    if (!o || !section || (n && (!keys || !values))) {
        psx::set_error("overview_add_section: bad arguments");
        return PSX_ERR_INVALID;
    }
    Xml e(section);
    for (size_t i = 0; i < n; ++i) e.kids.emplace_back(keys[i], values[i] ? values[i] : "");
    o->root.kids.push_back(std::move(e));
    return PSX_OK;
}

int psx_overview_add_misc_info(psx_overview* o, long long unix_time)
{
    if (!o) return PSX_ERR_INVALID;
    // OutputFileWriter::add_misc_info (output_stats.hpp:122-132)
    const std::time_t t = (std::time_t)unix_time;
    char buf[128];
    Xml e("misc_info");
    std::tm tm_l{}, tm_u{};
    localtime_r(&t, &tm_l);
    gmtime_r(&t, &tm_u);
    std::strftime(buf, sizeof buf, "%Y-%m-%d-%H:%M", &tm_l);
    e.kids.emplace_back("local_datetime", buf);
    std::strftime(buf, sizeof buf, "%Y-%m-%d-%H:%M", &tm_u);
    e.kids.emplace_back("utc_datetime", buf);
    o->root.kids.push_back(std::move(e));
    return PSX_OK;
}

int psx_overview_add_dm_list(psx_overview* o, const float* dms, size_t n)
{
    if (!o || (n && !dms)) return PSX_ERR_INVALID;
    // add_dm_list (output_stats.hpp:158-173): values with 4 decimals
    Xml e("dedispersion_trials");
    e.attrs["count"] = num((long long)n);
    for (size_t i = 0; i < n; ++i) {
        Xml t("trial", fixed4(dms[i]));
        t.attrs["id"] = num((long long)i);
        e.kids.push_back(std::move(t));
    }
    o->root.kids.push_back(std::move(e));
    return PSX_OK;
}

int psx_overview_add_acc_list(psx_overview* o, const float* accs, size_t n, float cdm)
{
    if (!o || (n && !accs)) return PSX_ERR_INVALID;
    // add_acc_list (output_stats.hpp:175-186)
    Xml e("acceleration_trials");
    e.attrs["count"] = num((long long)n);
    e.attrs["DM"] = fixed4(cdm);
    for (size_t i = 0; i < n; ++i) {
        Xml t("trial", num((double)accs[i]));
        t.attrs["id"] = num((long long)i);
        e.kids.push_back(std::move(t));
    }
    o->root.kids.push_back(std::move(e));
    return PSX_OK;
}

int psx_overview_add_device_info(psx_overview* o, int runtime_version, int driver_version,
                                 const int* ids, const char* const* names, const int* major,
                                 const int* minor, size_t n)
{
    if (!o || (n && (!ids || !names || !major || !minor))) return PSX_ERR_INVALID;
    // add_gpu_info (output_stats.hpp:141-156)
    Xml e("cuda_device_parameters");
    e.kids.emplace_back("runtime", num((long long)runtime_version));
    e.kids.emplace_back("driver", num((long long)driver_version));
    for (size_t i = 0; i < n; ++i) {
        Xml d("cuda_device");
        d.attrs["id"] = num((long long)ids[i]);
        d.kids.emplace_back("name", names[i] ? names[i] : "");
        d.kids.emplace_back("major_cc", num((long long)major[i]));
        d.kids.emplace_back("minor_cc", num((long long)minor[i]));
        e.kids.push_back(std::move(d));
    }
    o->root.kids.push_back(std::move(e));
    return PSX_OK;
}

int psx_overview_add_candidates(psx_overview* o, const psx_candidate* nodes, const int* sizes,
                                size_t n_nodes, const psx_candidate_score* scores,
                                const long long* byte_offsets)
{
    psx::clear_error();
    if (!o || (n_nodes && (!nodes || !sizes || !scores))) {
        psx::set_error("overview_add_candidates: bad arguments");
        return PSX_ERR_INVALID;
    }
    std::vector<size_t> roots;
    if (!forest_roots(sizes, n_nodes, &roots)) {
        psx::set_error("overview_add_candidates: subtree sizes do not describe a forest");
        return PSX_ERR_INVALID;
    }
    // add_candidates (output_stats.hpp:188-209); no folding: opt_period and
    // folded_snr stay 0 as in a run without folding
    Xml e("candidates");
    for (size_t q = 0; q < roots.size(); ++q) {
        const psx_candidate& c = nodes[roots[q]];
        const psx_candidate_score& s = scores[q];
        Xml x("candidate");
        x.attrs["id"] = num((long long)q);
        x.kids.emplace_back("period", num(1.0 / (double)c.freq));
        x.kids.emplace_back("opt_period", num(0.0));
        x.kids.emplace_back("dm", num((double)c.dm));
        x.kids.emplace_back("acc", num((double)c.acc));
        x.kids.emplace_back("nh", num((long long)c.nh));
        x.kids.emplace_back("snr", num((double)c.snr));
        x.kids.emplace_back("folded_snr", num(0.0));
        x.kids.emplace_back("is_adjacent", num((long long)s.is_adjacent));
        x.kids.emplace_back("is_physical", num((long long)s.is_physical));
        x.kids.emplace_back("ddm_count_ratio", num((double)s.ddm_count_ratio));
        x.kids.emplace_back("ddm_snr_ratio", num((double)s.ddm_snr_ratio));
        x.kids.emplace_back("nassoc", num((long long)(sizes[roots[q]] - 1)));
        x.kids.emplace_back("byte_offset", num(byte_offsets ? byte_offsets[q] : 0LL));
        e.kids.push_back(std::move(x));
    }
    o->root.kids.push_back(std::move(e));
    return PSX_OK;
}

int psx_overview_write(psx_overview* o, const char* path, char* h_text, size_t cap,
                       size_t* n_text)
{
    psx::clear_error();
    if (!o) return PSX_ERR_INVALID;
    std::string s = "<?xml version='1.0' encoding='ISO-8859-1'?>\n";
    o->root.write(s, 0);
    if (n_text) *n_text = s.size();
    if (h_text) {
        if (cap < s.size() + 1) {
            psx::set_error("overview_write: %zu bytes, buffer holds %zu", s.size() + 1, cap);
            return PSX_ERR_OVERFLOW;
        }
        std::memcpy(h_text, s.c_str(), s.size() + 1);
    }
    if (path) {
        FILE* f = std::fopen(path, "wb");
        if (!f) {
            psx::set_error("overview_write: cannot open %s", path);
            return PSX_ERR_IO;
        }
        const bool ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
        if (std::fclose(f) != 0 || !ok) {
            psx::set_error("overview_write: write to %s failed", path);
            return PSX_ERR_IO;
        }
    }
    return PSX_OK;
}

}  // extern "C"
