"""The FP32 CPU rendering (oracle/cpu_render.cpp), timed by the benchmark
as its CPU baseline, finds what the FP64 oracle finds: every candidate
whose S/N clears the threshold by more than 0.2 % in both, with identical
(acceleration, harmonic, frequency bin) and S/N within 1e-3 relative; the
result does not depend on the number of threads."""
import numpy as np
import pytest

from helpers import match_candidates


@pytest.fixture(scope="module")
def O():
    from oracle import oracle as O
    O.lib()
    O.cpu_render()
    return O


@pytest.mark.parametrize("n,survey", [(1 << 16, False), (1 << 17, True)])
def test_cpu_render_matches_oracle(O, n, survey):
    from peasoup_b200 import synth
    if survey:
        ts = 76e-6
        plan = synth.survey_plan(ndm=2, nsamps=n - 700, tsamp=ts, seed=3, npulsars=2, nbirdies=5)
        for ps in plan.pulsars:
            ps.amp = 40.0
        x = synth.survey_series_np(plan, 0, seed=3)
        extra = dict(birdie_freqs=plan.birdie_freqs, birdie_widths=plan.birdie_widths,
                     acc_lo=-100.0, acc_hi=100.0, nharmonics=5, min_snr=6.0)
    else:
        ts = 64e-6
        x = synth.make_series_np(synth.SeriesSpec(
            nsamps=n, tsamp=ts, pulsars=[synth.Pulsar(5.7e-3, 12.0, 0.05, 1.0)]), 0)
        extra = dict(acc_lo=-50.0, acc_hi=50.0, nharmonics=4, min_snr=7.0)
    p = O.SearchParams(fft_size=n, tsamp=ts, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ,
                       **extra)
    want, wtr = O.search_dm(x, p)
    got, gtr, sec = O.cpu_search_dm(x, p, 4)
    assert sec > 0
    nm, ua, ub, worst = match_candidates(got, want, p.min_snr)
    assert nm > 0 and not ua and not ub and worst < 1e-3, (ua[:3], ub[:3], worst)
    one, otr, _ = O.cpu_search_dm(x, p, 1)
    assert np.array_equal(one, got) and np.array_equal(otr, gtr)
