"""End to end on the GPU: a block of dedispersed series through the
product's Worker loop and post-search chain (peasoup_b200.pipeline) against
the reference's unmodified Worker (oracle/_ref, on the same GPU) followed by
its own DMDistiller, HarmonicDistiller, CandidateScorer and writers."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same_records(a, b):
    assert len(a) == len(b)
    for f in ("dm", "dm_idx", "acc", "nh", "freq"):
        assert np.array_equal(a[f], b[f]), f
    assert np.allclose(a["snr"], b["snr"], rtol=1e-5, atol=0)


def _records(blob, offsets, sizes):
    """Every record of a candidates.peasoup file, candidate by candidate."""
    from peasoup_b200.search import CAND_DTYPE
    out = []
    for off in offsets:
        k = int(np.frombuffer(blob, np.int32, count=1, offset=int(off))[0])
        out.append(np.frombuffer(blob, CAND_DTYPE, count=k, offset=int(off) + 4))
    return np.concatenate(out)


def test_search_to_outputs_matches_reference(cuda, psx, ref_gpu, ref_host):
    from peasoup_b200 import output, pipeline, search, synth
    O = ref_gpu
    n, ts = 1 << 16, 64e-6
    plan = synth.survey_plan(ndm=4, nsamps=n - 700, tsamp=ts, seed=8, npulsars=2, nbirdies=0)
    for p in plan.pulsars:
        p.amp = 40.0
    xs = np.stack([synth.survey_series_np(plan, d, seed=8) for d in range(4)])
    kw = dict(acc_lo=-60.0, acc_hi=60.0, nharmonics=4, min_snr=6.0)
    params = search.SearchParams(fft_size=n, tsamp=ts, cfreq_hz=synth.CFREQ_HZ,
                                 ch_bw_hz=synth.CH_BW_HZ, mode="plain", **kw)
    foff, nchans = -1.09, 64
    cfreq = synth.CFREQ_HZ / 1e6
    with tempfile.TemporaryDirectory() as d:
        nodes, sizes, scores, offsets, times = pipeline.search_to_outputs(
            xs, plan.dms, params, d, foff_mhz=foff, nchans=nchans, cfreq_mhz=cfreq, limit=50)
        mine = open(os.path.join(d, "candidates.peasoup"), "rb").read()
        xml = open(os.path.join(d, "overview.xml"), encoding="latin-1").read()
        # the reference: its Worker's per-DM trees, then its own classes
        op = O.SearchParams(fft_size=n, tsamp=ts, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ, **kw)
        rn, rs = O.ref_worker_search_forest(xs, ts, plan.dms, n, op)
        r1 = ref_host.ref_distill_forest(2, rn, rs, keep_related=True)
        rn2, rs2 = ref_host.ref_distill_forest(0, *r1, keep_related=True, fractional=False)
        rn2, rs2 = output.limit(rn2, rs2, 50)
        open(os.path.join(d, "ref.peasoup"), "wb").close()
        roff = ref_host.ref_write_binary(d, "ref.peasoup", rn2, rs2)
        theirs = open(os.path.join(d, "ref.peasoup"), "rb").read()
    # identical trees and candidate identities; S/N to the stated tolerance
    # (the two implementations reduce the spectrum statistics in different
    # orders, so S/N may differ in the last bits)
    assert len(output.roots(sizes)) > 3 and (sizes > 1).any()
    _same_records(nodes, rn2)
    assert np.array_equal(sizes, rs2) and np.array_equal(offsets, roff)
    assert len(mine) == len(theirs)
    _same_records(_records(mine, offsets, sizes), _records(theirs, roff, rs2))
    want = ref_host.ref_score_forest(rn2, rs2, ts, cfreq, foff, abs(foff) * nchans)
    for f in ("is_physical", "is_adjacent", "nassoc"):
        assert np.array_equal(scores[f], want[f])
    for f in ("ddm_count_ratio", "ddm_snr_ratio"):
        assert np.allclose(scores[f], want[f], rtol=1e-5, atol=0)
    assert xml.count("<candidate id=") == len(output.roots(sizes))
    assert "<dedispersion_trials count='4'>" in xml and "<acceleration_trials" in xml
