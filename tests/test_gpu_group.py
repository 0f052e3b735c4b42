"""Grouped prologues (psx_search_config.group_dms): the per-DM prologues of
several DM trials of one psx_search_block call run as one batch of
row-indexed launches and batched cuFFT plans.  Every row must be computed
exactly as the per-DM prologue computes it, so the dereddened series, its
statistics and every candidate (S/N bits included) must equal the
ungrouped call's.  Covered: a partial last group, zero padding
(nsamps < fft_size), birdies, host and device series, the default rule
(4 rows when DM trials average at most 32 acceleration trials), profiling
and the record-buffer growth retry of a grouped slot.
"""
import numpy as np
import pytest

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


def _block(S, n, ts, nsamps, ndm, seed, **kw):
    search, synth = S
    xs = np.stack([synth.make_series_np(synth.SeriesSpec(
        nsamps=nsamps, tsamp=ts,
        pulsars=[synth.Pulsar(3.1e-3 * (d % 5 + 1), 6.0 * (d % 3), 0.05, 0.7)]), seed + d)
        for d in range(ndm)])
    dms = np.linspace(0.0, 40.0, ndm).astype(np.float32)
    return xs, dms


def _run(S, n, ts, xs, dms, group, device=False, **kw):
    search, _ = S
    s = search.AccelSearch(_params(S, n, ts, group_dms=group, **kw))
    if device:
        import torch
        xs = torch.from_numpy(xs).cuda()
    out = s.search_block(xs, dms)
    info = s.info()
    tap = s.debug_tap(0)
    s.close()
    return out, info, tap


def _equal(a, b):
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("n,nsamps,lanes", [(1 << 20, 1 << 20, 1), (1 << 20, 900_000, 1),
                                            (3 << 18, 3 << 18, 1), (1 << 20, 1 << 20, 2),
                                            (1 << 17, 1 << 17, 1)])
def test_grouped_equals_per_dm(S, n, nsamps, lanes):
    """(2^17 points: the trials on cuFFT's complex transform; lanes 2: launch
    groups alternate over two streams.)"""
    ts = 64e-6
    xs, dms = _block(S, n, ts, nsamps, 11, 40)
    kw = dict(acc_lo=-20.0, acc_hi=20.0, nharmonics=4, min_snr=7.0, batch=8, lanes=lanes,
              birdie_freqs=np.array([50.0, 123.4], np.float32),
              birdie_widths=np.array([0.5, 1.0], np.float32))
    ref, info0, tap0 = _run(S, n, ts, xs, dms, 1, **kw)
    assert info0["group_dms"] == 0
    assert len(ref[0]) > 0
    got, info4, tap4 = _run(S, n, ts, xs, dms, 4, **kw)  # groups of 4, 4 and 3
    assert info4["group_dms"] == 4
    _equal(ref, got)
    # the last DM trial's dereddened series and (mean*N, std*N), bit for bit
    assert np.array_equal(tap0[0], tap4[0]) and np.array_equal(tap0[3], tap4[3])
    got_d, info_d, _ = _run(S, n, ts, xs, dms, 4, device=True, **kw)
    assert info_d["group_dms"] == 4
    _equal(ref, got_d)


def test_default_rule_and_profile(S):
    search, _ = S
    n, ts = 1 << 20, 64e-6
    xs, dms = _block(S, n, ts, n, 10, 60)
    kw = dict(acc_lo=-10.0, acc_hi=10.0, nharmonics=3, min_snr=7.0, batch=8)
    ref, _, _ = _run(S, n, ts, xs, dms, 1, **kw)
    s = search.AccelSearch(_params(S, n, ts, **kw))
    s.set_profile(True)
    got = s.search_block(xs, dms)
    info = s.info()
    prof = s.profile(reset=True)
    assert info["group_dms"] == 4  # 10 DM trials of a few acceleration trials each
    _equal(ref, got)
    assert prof["dms"] == 10 and prof["prologue_ms"] > 0 and prof["harm_ms"] > 0
    # a call with no more DM trials than a group holds runs them one by one
    s.search_block(xs[:4], dms[:4])
    assert s.info()["group_dms"] == 0
    s.close()
    # many acceleration trials per DM trial (about 53 at 512 us sampling,
    # +-300 m/s^2): the default does not group
    s = search.AccelSearch(_params(S, n, 512e-6, acc_lo=-300.0, acc_hi=300.0, nharmonics=3,
                                   min_snr=7.0, batch=8))
    s.search_block(xs, dms)
    assert s.info()["group_dms"] == 0 and s.info()["ntrials"] > 32 * 10
    s.close()


def test_grouped_record_growth(S):
    """A threshold of zero overflows the first record buffers (2^20 records
    of a chunk's trial list, 2^18 of a grouped slot): the trials run again
    with a larger buffer, and the result is as if they had run once."""
    n, ts = 1 << 19, 64e-6
    xs, dms = _block(S, n, ts, n, 5, 80)
    kw = dict(acc_lo=-30.0, acc_hi=30.0, nharmonics=4, min_snr=0.0, batch=8)
    ref, info0, _ = _run(S, n, ts, xs, dms, 1, **kw)
    assert info0["above_threshold"] > 5 * (1 << 20)  # over 2^21 per chunk of two
    got, info2, _ = _run(S, n, ts, xs, dms, 2, **kw)
    assert info2["group_dms"] == 2
    _equal(ref, got)
