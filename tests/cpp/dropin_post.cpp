// dropin_post.cpp -- the reference's steps after its Workers
// (src/pipeline_multi.cu:531-587) written against the drop-in classes:
// DMDistiller and HarmonicDistiller with association trees,
// CandidateScorer, --limit, CandidateFileWriter and OutputFileWriter.
//
//   dropin_post <in.bin> <outdir> <limit> <tsamp> <cfreq> <foff> <bw>
//
// in.bin: int32 number of DM trials, then per DM trial an int32 count and
// that many 24-byte records, its acceleration-distilled candidate forest
// (nodes in depth-first order) followed by int32 subtree sizes.  Writes
// outdir/candidates.peasoup and outdir/overview.xml (DM list 0, 0.5, ...,
// acceleration list {0}, candidates, so that it compares with the
// reference's writer fed the same).
#include <cstdio>
#include <cstdlib>
#include <map>
#include <vector>
#include "data_types/candidates.hpp"
#include "transforms/distiller.hpp"
#include "transforms/scorer.hpp"
#include "utils/output_stats.hpp"

int main(int argc, char** argv)
{
    if (argc != 8) {
        std::fprintf(stderr, "usage: dropin_post in.bin outdir limit tsamp cfreq foff bw\n");
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int ndm = 0;
    if (std::fread(&ndm, sizeof(int), 1, f) != 1) return 2;
    CandidateCollection dm_cands;
    for (int d = 0; d < ndm; ++d) {
        int n = 0;
        if (std::fread(&n, sizeof(int), 1, f) != 1) return 2;
        std::vector<psx_candidate> nodes(n);
        std::vector<int> sizes(n);
        if (n && (std::fread(nodes.data(), sizeof(psx_candidate), n, f) != (size_t)n ||
                  std::fread(sizes.data(), sizeof(int), n, f) != (size_t)n))
            return 2;
        dm_cands.append(from_forest(nodes.data(), sizes.data(), nodes.size()));
    }
    std::fclose(f);
    const int limit = std::atoi(argv[3]);
    const float tsamp = (float)std::atof(argv[4]), cfreq = (float)std::atof(argv[5]),
                foff = (float)std::atof(argv[6]), bw = (float)std::atof(argv[7]);
    const float freq_tol = 1e-4f, max_harm = 16.0f;

    DMDistiller dm_still(freq_tol, true);
    HarmonicDistiller harm_still(freq_tol, max_harm, true, false);
    dm_cands.cands = dm_still.distill(dm_cands.cands);
    dm_cands.cands = harm_still.distill(dm_cands.cands);
    CandidateScorer cand_scorer(tsamp, cfreq, foff, bw);
    cand_scorer.score_all(dm_cands.cands);
    if ((int)dm_cands.cands.size() > limit) dm_cands.cands.resize(limit);

    CandidateFileWriter cand_files(argv[2]);
    cand_files.write_binary(dm_cands.cands, "candidates.peasoup");
    OutputFileWriter stats;
    std::vector<float> dms;
    for (int d = 0; d < ndm; ++d) dms.push_back(0.5f * d);
    stats.add_dm_list(dms);
    std::vector<float> accs(1, 0.0f);
    stats.add_acc_list(accs, 0.0f);
    stats.add_candidates(dm_cands.cands, cand_files.byte_mapping);
    stats.to_file(std::string(argv[2]) + "/overview.xml");
    std::printf("%zu\n", dm_cands.cands.size());
    return 0;
}
