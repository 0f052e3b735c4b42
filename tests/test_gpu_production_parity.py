"""Candidate parity of the production configuration at the benchmark sizes.

The headline throughput is measured on one configuration of the engine:
the batched mode with the library's two-pass transform (resample gather in
pass 1, ``fft_form`` 3), the three-trial harmonic kernel (shape 6), launch
groups of 96 trials and CUDA-graph schedules.  These tests run exactly that
configuration (and the autotuner's pick) on the survey workload at 2^23
points and on the small plain workload at 2^20, and compare its candidates
with

  * the reference's unmodified ``Worker::start`` (src/pipeline_multi.cu:
    161-294, built from its own sources into oracle/_ref) on the same
    series and zap list: the per-DM acceleration-distilled lists;
  * the FP64 oracle on chosen acceleration trials of the same DM trials:
    the per-trial harmonic-distilled lists.

The agreement asked for is bit-exact (dm, acc, nh, bin) sets with S/N
within 1e-3 relative.  The spectra of two FP32 transforms differ by about
1e-6 of their RMS, so a peak whose S/N lies within that distance of the
threshold can be above it in one and below it in the other.  Every such
"flip" is counted, printed and required to lie within FLIP_MARGIN of the
threshold (relative); the count itself is asserted small.
"""
import os
import tempfile

import numpy as np
import pytest

from helpers import cand_key

pytestmark = pytest.mark.gpu

N_SURVEY = 1 << 23
TS_SURVEY = 76e-6
# Relative distance from the threshold within which a candidate may be
# present in one list and absent from the other.
FLIP_MARGIN_REF = 1e-4      # FP32 engine vs the reference's FP32 Worker
FLIP_MARGIN_ORACLE = 2e-3   # FP32 engine vs the FP64 oracle
MAX_FLIPS = 4
SNR_RTOL = 1e-3


def flip_report(got, want, thresh, margin, label):
    """Compares two candidate lists by (dm_idx, acc, nh, freq).  Returns
    (n_matched, flips, worst relative S/N difference of the matched pairs);
    prints every flip with its distance from the threshold."""
    ga = {cand_key(c): float(c["snr"]) for c in got}
    wa = {cand_key(c): float(c["snr"]) for c in want}
    matched = set(ga) & set(wa)
    worst = max((abs(ga[k] - wa[k]) / abs(wa[k]) for k in matched), default=0.0)
    flips = [("engine", k, ga[k]) for k in ga if k not in wa]
    flips += [("other", k, wa[k]) for k in wa if k not in ga]
    print(f"{label}: {len(matched)} matched, {len(flips)} flips, worst S/N rel {worst:.2e}")
    for side, k, s in flips:
        print(f"  flip only in {side}: {k} snr {s:.6f} ({(s / thresh - 1):+.2e} from threshold)")
    bad = [f for f in flips if abs(f[2] / thresh - 1) > margin]
    assert not bad, (label, bad[:5])
    assert len(flips) <= MAX_FLIPS, (label, len(flips))
    return len(matched), flips, worst


@pytest.fixture(scope="module")
def S(cuda, psx):
    from peasoup_b200 import search, synth
    return search, synth


@pytest.fixture(scope="module")
def survey(S):
    """Config 2's survey series at 2^23 for three DM trials: the DM trials
    of two injected pulsars and one without."""
    search, synth = S
    plan = synth.survey_plan(ndm=256, nsamps=N_SURVEY, tsamp=TS_SURVEY)
    picks = [int(plan.pulsar_dm_idx[0]), int(plan.pulsar_dm_idx[1]), 0]
    xs = np.stack([synth.survey_series_np(plan, d) for d in picks])
    dms = plan.dms[picks]
    fd, zap = tempfile.mkstemp(suffix=".txt")
    with os.fdopen(fd, "w") as f:
        f.write(plan.zaplist_text())
    yield plan, picks, xs, dms, zap
    os.unlink(zap)


def _survey_params(S, plan, **kw):
    search, synth = S
    p = dict(fft_size=N_SURVEY, tsamp=TS_SURVEY, acc_lo=-100.0, acc_hi=100.0, nharmonics=5,
             min_snr=9.0, cfreq_hz=synth.CFREQ_HZ, ch_bw_hz=synth.CH_BW_HZ,
             birdie_freqs=plan.birdie_freqs, birdie_widths=plan.birdie_widths)
    p.update(kw)
    return search.SearchParams(**p)


def _oracle_params(oracle, synth, n, ts, **kw):
    p = dict(fft_size=n, tsamp=ts, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ)
    p.update(kw)
    return oracle.SearchParams(**p)


@pytest.fixture(scope="module")
def production(S, survey):
    """The benchmark's configuration on the three survey DM trials: per-DM
    lists and per-trial lists."""
    search, synth = S
    plan, picks, xs, dms, _ = survey
    s = search.AccelSearch(_survey_params(S, plan, mode="batched", batch=96, harm_shape=6,
                                          graph=True))
    per_dm = s.search_block(xs, dms, per_dm=True)
    per_trial = s.search_block(xs, dms, per_dm=False)
    info = s.info()
    s.close()
    assert info["fft_form"] == 3 and info["harm_shape"] == 6 and info["graph"] == 1, info
    assert info["batch"] == 96, info
    return per_dm, per_trial


def test_survey_production_vs_reference_worker(S, survey, production, ref_gpu):
    """Config 2 at 2^23: the per-DM acceleration-distilled lists of the
    production configuration against the reference's own Worker."""
    search, synth = S
    plan, picks, xs, dms, zap = survey
    p = _oracle_params(ref_gpu, synth, N_SURVEY, TS_SURVEY, acc_lo=-100.0, acc_hi=100.0,
                       nharmonics=5, min_snr=9.0)
    rc, rna = ref_gpu.ref_worker_search(xs, TS_SURVEY, dms, N_SURVEY, p, zap)
    got = production[0][0]
    assert len(rc) > 0 and len(got) > 0
    nm, flips, worst = flip_report(got, rc, 9.0, FLIP_MARGIN_REF, "survey 2^23 vs reference")
    assert nm >= 0.95 * len(rc) and worst < SNR_RTOL
    # the two pulsars' DM trials carry a candidate at the pulsar's spin
    # frequency or a harmonic of it
    for pos in (0, 1):
        ps = plan.pulsars[pos]
        c = got[got["dm_idx"] == pos]
        r = c["freq"] * ps.period
        assert np.any((np.abs(r - np.round(r)) < 2e-3) & (np.round(r) >= 1)), (pos, c[:5])


def test_survey_production_vs_oracle(S, survey, production, oracle):
    """Config 2 at 2^23: per-trial lists of the production configuration
    against the FP64 oracle at acceleration 0 and at the grid trial nearest
    each injected pulsar's acceleration."""
    search, synth = S
    from peasoup_b200.transforms import AccelerationPlan
    plan, picks, xs, dms, _ = survey
    cands, _, trial, dmpos = production[1]
    for pos, d in enumerate(picks):
        accs = AccelerationPlan(-100.0, 100.0, 1.10, 64e-6, N_SURVEY, TS_SURVEY, synth.CFREQ_HZ,
                                synth.CH_BW_HZ).generate_accel_list(float(dms[pos]), 0.0)
        a_true = plan.pulsars[pos].accel if pos < 2 else 37.0
        a = float(accs[np.argmin(np.abs(accs - a_true))])
        # an equal acceleration range gives the one-trial list {acc}
        # (include/utils/utils.hpp:210-213)
        want = np.concatenate([oracle.search_dm(xs[pos], _oracle_params(
            oracle, synth, N_SURVEY, TS_SURVEY, dm=float(dms[pos]), dm_idx=pos, acc_lo=acc,
            acc_hi=acc, nharmonics=5, min_snr=9.0, birdie_freqs=plan.birdie_freqs,
            birdie_widths=plan.birdie_widths))[0] for acc in (0.0, a)])
        sel = (dmpos == pos) & np.isin(cands["acc"], np.float32([0.0, a]))
        assert set(np.unique(want["acc"])) <= {np.float32(0.0), np.float32(a)}
        nm, flips, worst = flip_report(cands[sel], want, 9.0, FLIP_MARGIN_ORACLE,
                                       f"survey 2^23 DM {d} acc 0/{a:.3f} vs oracle")
        assert worst < SNR_RTOL
        # the pulsars' DM trials have candidates; the noise-only one may have none
        assert nm > 0 if pos < 2 else nm == len(want) == int(sel.sum())


def test_survey_autotuned_equals_production(S, survey, production):
    """The autotuner's pick (launch group size and harmonic shape) changes
    grouping only: its per-DM lists equal the fixed production
    configuration's bit for bit."""
    search, synth = S
    plan, picks, xs, dms, _ = survey
    p = _survey_params(S, plan)
    t = search.autotune(p, batches=(32, 64, 96, 128), reps=1, max_trials=128)
    import dataclasses
    s = search.AccelSearch(dataclasses.replace(p, batch=t["batch"], harm_shape=t["harm_shape"]))
    got = s.search_block(xs, dms, per_dm=True)
    assert s.info()["fft_form"] == 3
    s.close()
    for a, b in zip(got, production[0]):
        assert np.array_equal(a, b), t


def test_config1_plain_and_production_vs_oracle_and_reference(S, oracle, ref_gpu):
    """Config 1 at its stated size (2^20 points, 64 us, -50..50 m/s^2, 4
    folds, S/N 7, one trial per launch): the plain mode and the production
    configuration against the FP64 oracle (whole DM trial, per-trial lists)
    and against the reference's Worker (per-DM lists); the known answer is
    the injected 175.44 Hz pulsar, strongest at the trial nearest +12."""
    search, synth = S
    n, ts = 1 << 20, 64e-6
    x = synth.config1_series(0)
    kw = dict(acc_lo=-50.0, acc_hi=50.0, nharmonics=4, min_snr=7.0)
    want, _ = oracle.search_dm(x, _oracle_params(oracle, synth, n, ts, **kw))
    rc, _ = ref_gpu.ref_worker_search(x[None, :], ts, np.zeros(1, np.float32), n,
                                      _oracle_params(ref_gpu, synth, n, ts, **kw), "")
    f0 = 1 / 5.7e-3
    for mode, extra in (("plain", {}), ("batched", dict(batch=96, harm_shape=6, graph=True))):
        s = search.AccelSearch(search.SearchParams(fft_size=n, tsamp=ts, mode=mode,
                                                   cfreq_hz=synth.CFREQ_HZ,
                                                   ch_bw_hz=synth.CH_BW_HZ, **kw, **extra))
        trials, _, _ = s.search(x, 0.0, 0, per_dm=False)
        per_dm, _, _ = s.search(x, 0.0, 0, per_dm=True)
        info = s.info()
        s.close()
        if mode == "batched":
            assert info["fft_form"] == 3 and info["harm_shape"] == 6
        nm, _, worst = flip_report(trials, want, 7.0, FLIP_MARGIN_ORACLE,
                                   f"config 1 {mode} vs oracle")
        assert nm > 0 and worst < SNR_RTOL
        nm, _, worst = flip_report(per_dm, rc, 7.0, FLIP_MARGIN_REF,
                                   f"config 1 {mode} vs reference")
        assert nm == len(rc) and worst < SNR_RTOL
        best = trials[np.argmax(trials["snr"])]
        assert abs(best["freq"] / f0 - 1) < 1e-4 and best["acc"] == 0.0, best


def test_config1_block_grouped_vs_reference(S, ref_gpu):
    """Config 1's statistics over 10 DM trials in one block call: with about
    3 acceleration trials per DM trial the engine groups the prologues by 4
    (batched cuFFT plans, row-indexed prologue kernels); its per-DM lists
    against the reference's Worker over the same 10 series, and bit for bit
    against the same block without grouping."""
    search, synth = S
    n, ts, ndm = 1 << 20, 64e-6, 10
    xs = np.stack([synth.config1_series(d) for d in range(ndm)])
    dms = (0.5 * np.arange(ndm)).astype(np.float32)
    kw = dict(acc_lo=-50.0, acc_hi=50.0, nharmonics=4, min_snr=7.0)
    rc, _ = ref_gpu.ref_worker_search(xs, ts, dms, n, _oracle_params(ref_gpu, synth, n, ts, **kw),
                                      "")
    outs = []
    for group in (0, 1):
        s = search.AccelSearch(search.SearchParams(fft_size=n, tsamp=ts, cfreq_hz=synth.CFREQ_HZ,
                                                   ch_bw_hz=synth.CH_BW_HZ, batch=96,
                                                   harm_shape=6, group_dms=group, **kw))
        c, na, tr, dm = s.search_block(xs, dms, per_dm=True)
        info = s.info()
        s.close()
        assert info["group_dms"] == (4 if group == 0 else 0)
        outs.append((c, na, dm))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)
    nm, _, worst = flip_report(outs[0][0], rc, 7.0, FLIP_MARGIN_REF,
                               "config 1 block, grouped prologues, vs reference")
    assert nm == len(rc) and nm >= ndm and worst < SNR_RTOL
