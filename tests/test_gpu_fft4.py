"""The batched path's own transform (fft_form 3: the resample gather in the
first of two passes of a four-step complex transform of the series read as
interleaved pairs, then the unpack + interbin + normalise kernel):

  * the normalised interbinned spectrum of tapped trials against FP64
    (numpy's real transform of the same resampled series) within 1e-5
    relative, |a - b| <= 1e-5 (|b| + RMS), at every row length the two
    passes support and for every row count (768 for 3 * 2^k, 1024, and
    2048 / 4096 for the long segments of 2^26 / 2^27 points);
  * candidate lists identical to cuFFT's complex transform (fft_form 1) and
    to the reference's real transform (plain mode), S/N within 1e-5.
"""
import numpy as np
import pytest

from helpers import err_vs_mag_or_rms, match_candidates

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S(cuda, psx):
    from peasoup_b200 import search, synth
    return search, synth


def _params(S, n, tsamp, **kw):
    search, synth = S
    p = dict(fft_size=n, tsamp=tsamp, cfreq_hz=synth.CFREQ_HZ, ch_bw_hz=synth.CH_BW_HZ)
    p.update(kw)
    return search.SearchParams(**p)


def _fp64_spectrum(tim, idx, norm2):
    """Interbinned, normalised spectrum of tim[idx] in FP64 (the reference's
    forming and normalising steps, src/kernels.cu:238-259 and :496-507)."""
    x = tim[idx.astype(np.int64)].astype(np.float64)
    X = np.fft.rfft(x)
    prev = np.concatenate([[0j], X[:-1]])
    amp = np.sqrt(np.maximum(np.abs(X) ** 2, 0.5 * np.abs(X - prev) ** 2))
    return (amp - float(norm2[0])) / float(norm2[1])


@pytest.mark.parametrize("n", [1 << 19, 1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25,
                               3 << 17, 3 << 20, 3 << 23])
def test_spectrum_vs_fp64(S, oracle, n):
    search, synth = S
    ts = 64e-6
    logn = n.bit_length()
    x = synth.make_series_np(synth.SeriesSpec(
        nsamps=n, tsamp=ts, pulsars=[synth.Pulsar(4.1e-3, 35.0, 0.04, 0.5)]), logn)
    s = search.AccelSearch(_params(S, n, ts, batch=4, acc_lo=-40.0, acc_hi=40.0,
                                   nharmonics=2, min_snr=9.0))
    s.search(x, 0.0, 0, per_dm=False)
    assert s.info()["fft_form"] == 3
    from peasoup_b200.transforms import AccelerationPlan
    accs = AccelerationPlan(-40.0, 40.0, 1.10, 64e-6, n, ts, synth.CFREQ_HZ,
                            synth.CH_BW_HZ).generate_accel_list(0.0, 0.0)
    for t in sorted({0, len(accs) // 2, len(accs) - 1}):
        tim, tr, ps, norm2 = s.debug_tap(t)
        idx = oracle.resampleII_index(n, float(accs[t]), ts)
        want = _fp64_spectrum(tim, idx, norm2)
        err = err_vs_mag_or_rms(ps, want)
        assert err < 1e-5, (logn, t, err)
    s.close()


@pytest.mark.parametrize("n,acc", [(1 << 26, 0.05), (1 << 27, 0.02)])
def test_long_segment_vs_fp64_and_plain(S, oracle, n, acc):
    """Long segments (2^26 and 2^27 points, tsamp 64 us: 1.2 and 2.4 h) on
    the two-pass transform with 2048- and 4096-row columns: the normalised
    spectrum of the first and last trial against FP64 (within 1e-5, as at
    the shorter lengths), and the candidates against the plain path (the
    reference's cuFFT real transform, include/transforms/ffter.hpp:54-80),
    S/N within 1e-5.  A narrow acceleration range keeps the trial count
    small (the step shrinks as 1/tobs^2)."""
    import torch
    search, synth = S
    ts = 64e-6
    g = torch.Generator(device="cuda").manual_seed(n.bit_length())
    x = torch.randn(n, device="cuda", generator=g)
    t = torch.arange(n, device="cuda", dtype=torch.float64)
    k = 0.01 * ts / (2.0 * 299792458.0)
    ph = torch.frac((t - k * t * (t - n)) * ts / 9.7e-3)
    x += (0.05 * torch.exp(-0.5 * ((ph - 0.5) / 0.02) ** 2)).float()
    del t, ph
    kw = dict(acc_lo=-acc, acc_hi=acc, nharmonics=5, min_snr=7.0)
    s = search.AccelSearch(_params(S, n, ts, batch=4, **kw))
    own = s.search(x, 0.0, 0, per_dm=False)[0]
    assert s.info()["fft_form"] == 3
    from peasoup_b200.transforms import AccelerationPlan
    accs = AccelerationPlan(-acc, acc, 1.10, 64e-6, n, ts, synth.CFREQ_HZ,
                            synth.CH_BW_HZ).generate_accel_list(0.0, 0.0)
    assert 2 <= len(accs) <= 16
    for tr_i in sorted({0, len(accs) - 1}):
        tim, tr, ps, norm2 = s.debug_tap(tr_i)
        idx = oracle.resampleII_index(n, float(accs[tr_i]), ts)
        assert np.array_equal(tr, tim[idx.astype(np.int64)])
        err = err_vs_mag_or_rms(ps, _fp64_spectrum(tim, idx, norm2))
        del tim, tr, idx
        assert err < 1e-5, (n, tr_i, err)
    s.close()
    p = search.AccelSearch(_params(S, n, ts, mode="plain", **kw))
    plain = p.search(x, 0.0, 0, per_dm=False)[0]
    p.close()
    assert len(own) > 3
    nm, ua, ub, worst = match_candidates(own, plain, 7.0, margin=1e-4)
    assert not ua and not ub and worst < 1e-5, (ua[:3], ub[:3], worst)
    f0 = 1 / 9.7e-3
    r = own["freq"] / f0
    assert np.any(np.abs(r - np.round(r)) < 1e-4)


@pytest.mark.parametrize("n", [1 << 20, 1 << 22, 3 << 20])
def test_candidates_match_cufft_paths(S, n):
    search, synth = S
    ts = 64e-6
    x = synth.make_series_np(synth.SeriesSpec(
        nsamps=n, tsamp=ts, pulsars=[synth.Pulsar(3.3e-3, -25.0, 0.05, 0.4),
                                     synth.Pulsar(0.21, 4.0, 0.03, 0.6)]), 7)
    kw = dict(acc_lo=-60.0, acc_hi=60.0, nharmonics=4, min_snr=6.5)
    outs = {}
    for name, mode, form in (("own", "batched", 3), ("cufft", "batched", 1),
                             ("plain", "plain", 0)):
        s = search.AccelSearch(_params(S, n, ts, mode=mode, fft_form=form, batch=8, **kw))
        outs[name] = s.search(x, 2.0, 5, per_dm=False)[0]
        if mode == "batched":
            assert s.info()["fft_form"] == form
        s.close()
    assert len(outs["own"]) > 3
    for other in ("cufft", "plain"):
        nm, ua, ub, worst = match_candidates(outs["own"], outs[other], 6.5, margin=1e-4)
        assert not ua and not ub and worst < 1e-5, (other, ua[:3], ub[:3], worst)


def test_default_form_by_size(S):
    search, synth = S
    ts = 64e-6
    for n, want in ((1 << 16, 1), (3 << 16, 1), (1 << 19, 3), (3 << 17, 3)):
        s = search.AccelSearch(_params(S, n, ts, batch=2, acc_lo=-1.0, acc_hi=1.0,
                                       nharmonics=1, min_snr=9.0))
        s.search(synth.make_series_np(synth.SeriesSpec(nsamps=n, tsamp=ts), 2), 0.0, 0,
                 per_dm=False)
        assert s.info()["fft_form"] == want, n
        s.close()


@pytest.mark.parametrize("n", [1 << 19, 1 << 22, 3 << 19])
def test_gathered_series_bit_exact(S, oracle, n):
    """What pass 1 gathers (dumped by the debug tap instead of transformed)
    is the resampled series, bit for bit, against the oracle's FP64 index on
    the product's own dereddened series."""
    search, synth = S
    ts = 64e-6
    x = synth.make_series_np(synth.SeriesSpec(nsamps=n, tsamp=ts), 11)
    s = search.AccelSearch(_params(S, n, ts, batch=4, acc_lo=-300.0, acc_hi=300.0,
                                   nharmonics=2, min_snr=9.0))
    s.search(x, 0.0, 0, per_dm=False)
    assert s.info()["fft_form"] == 3
    from peasoup_b200.transforms import AccelerationPlan
    accs = AccelerationPlan(-300.0, 300.0, 1.10, 64e-6, n, ts, synth.CFREQ_HZ,
                            synth.CH_BW_HZ).generate_accel_list(0.0, 0.0)
    for t in sorted({0, len(accs) // 3, len(accs) - 1}):
        tim, tr, ps, _ = s.debug_tap(t)
        want = tim[oracle.resampleII_index(n, float(accs[t]), ts).astype(np.int64)]
        assert np.array_equal(tr, want), t
    s.close()


def test_padding_zap_lanes_graphs(S):
    """The two-pass path on a series shorter than the transform (zero
    padding) with a birdie list: one or two lanes, with or without graph
    capture, give bit-identical candidates (the same kernels in the same
    order), and those equal the plain path's (the reference's real
    transform), S/N within 1e-5."""
    search, synth = S
    n, ts = 1 << 19, 76e-6
    plan = synth.survey_plan(ndm=1, nsamps=n - 20000, tsamp=ts, seed=5, npulsars=2, nbirdies=5)
    for ps in plan.pulsars:
        ps.amp = 30.0
    x = synth.survey_series_np(plan, 0, seed=5)
    assert x.size == n - 20000
    kw = dict(acc_lo=-100.0, acc_hi=100.0, nharmonics=5, min_snr=6.0,
              birdie_freqs=plan.birdie_freqs, birdie_widths=plan.birdie_widths)
    outs = []
    for lanes, graph in ((1, True), (2, True), (2, False)):
        s = search.AccelSearch(_params(S, n, ts, batch=4, lanes=lanes, graph=graph, **kw))
        c = s.search(x, float(plan.dms[0]), 0, per_dm=False)[0]
        assert s.info()["fft_form"] == 3
        outs.append(c)
        s.close()
    assert len(outs[0]) > 3
    for c in outs[1:]:
        assert np.array_equal(c, outs[0])
    p = search.AccelSearch(_params(S, n, ts, mode="plain", **kw))
    cp = p.search(x, float(plan.dms[0]), 0, per_dm=False)[0]
    p.close()
    nm, ua, ub, worst = match_candidates(outs[0], cp, 6.0, margin=1e-4)
    assert nm > 3 and not ua and not ub and worst < 1e-5, (ua[:3], ub[:3], worst)
