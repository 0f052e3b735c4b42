"""The CPU oracle pinned against the reference (no GPU needed).

Golden sources:
  * tests/golden/host_golden.npz (make_host_golden.py): the acceleration
    list shipped in the reference's example_output/overview.xml, and
    outputs of the reference's own AccelerationPlan and distillers built
    from its sources;
  * tests/golden/ref_golden.npz (make_ref_golden.py, produced on a B200 by
    the reference's own CUDA build), when present: resampler index maps,
    FFTs, spectrum forming, running median, dereddening, zapping,
    statistics, harmonic sums, peak finding and whole Worker runs.
Plus textbook checks of the FP64 transforms against numpy.
"""
import os

import numpy as np
import pytest

from helpers import err_vs_rms, match_candidates, rel_err

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def hg():
    return np.load(os.path.join(GOLD, "host_golden.npz"))


@pytest.fixture(scope="module")
def rg():
    p = os.path.join(GOLD, "ref_golden.npz")
    if not os.path.exists(p):
        pytest.skip("reference GPU fixtures not generated yet")
    return np.load(p)


# ------------------------------------------------------------ transforms
@pytest.mark.parametrize("n", [16, 48, 1024, 3 << 10, 1 << 16, 3 << 14])
def test_fft_against_numpy(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    X = oracle.rfft(x)
    assert np.max(np.abs(X - np.fft.rfft(x))) < 1e-12 * np.sqrt(n) * np.max(np.abs(x)) * 10
    y = oracle.irfft(np.fft.rfft(x), n)
    assert np.allclose(y, n * x, rtol=0, atol=1e-9 * n)


def test_fft_rejects_unsupported_sizes(oracle):
    with pytest.raises(ValueError):
        oracle.rfft(np.zeros(5 * 64))


# ------------------------------------------------------------ acceleration plan
def test_accel_list_matches_overview_xml(oracle, hg):
    a = hg["overview_args"]
    got = oracle.accel_list(a[0], a[1], a[2], a[3], int(hg["overview_nsamps"]), a[4], a[5], a[6],
                            54.5, 54.5)
    want = hg["overview_accels"]
    assert got.size == want.size == 10758
    assert np.array_equal(got, want)


def _accel_cases(hg):
    cases, dms = hg["accel_cases"], hg["accel_dms"]
    vals = hg["accel_values"]
    for ci, dm, off, n in hg["accel_index"]:
        c = cases[int(ci)]
        args = (c[0], c[1], c[2], c[3], int(c[4]), c[5], c[6], c[7])
        yield args, float(dm), float(c[8]), vals[int(off):int(off) + int(n)]


def test_accel_list_matches_reference_plan(oracle, hg):
    k = 0
    for args, dm, cdm, want in _accel_cases(hg):
        got = oracle.accel_list(*args, dm, cdm)
        assert np.array_equal(got, want), (args, dm)
        k += 1
    assert k >= 30


def test_accel_list_live_reference(ref_host, oracle):
    rng = np.random.default_rng(1)
    for _ in range(40):
        lo = float(np.float32(-rng.uniform(0, 400)))
        hi = float(np.float32(rng.uniform(0, 400)))
        args = (lo, hi, float(np.float32(rng.uniform(1.01, 1.5))), 64e-6,
                int(2 ** rng.integers(18, 26)), float(np.float32(rng.uniform(32e-6, 256e-6))),
                1.4e9, 1.0e6)
        dm, cdm = float(np.float32(rng.uniform(0, 300))), float(np.float32(rng.uniform(0, 300)))
        assert np.array_equal(oracle.accel_list(*args, dm, cdm),
                              oracle.ref_accel_list(*args, dm, cdm))


# ------------------------------------------------------------ distillers
@pytest.mark.parametrize("name,kind", [("harm", 0), ("harm_related", 0), ("accel", 1), ("dm", 2)])
def test_distillers_match_reference(oracle, hg, name, kind):
    for j in range(4):
        c = hg[f"distill_{name}_{j}_in"]
        want = hg[f"distill_{name}_{j}_out"]
        wna = hg[f"distill_{name}_{j}_nassoc"]
        if kind == 0:
            frac = name == "harm"
            surv, arr, keep, na = oracle.harmonic_distill(c, 1e-4, 16.0, frac)
        elif kind == 1:
            surv, arr, keep, na = oracle.accel_distill(c, 637.5, 1e-4)
        else:
            surv, arr, keep, na = oracle.dm_distill(c, 1e-4)
        assert np.array_equal(surv, want), (name, j)
        if name != "harm":  # keep_related runs: association counts
            assert np.array_equal(na[keep == 1], wna), (name, j)


# ------------------------------------------------------------ stage checks
def test_median_and_stretch_basics(oracle):
    rng = np.random.default_rng(0)
    x = rng.standard_normal(5 * 1000 + 3)
    m = oracle.median_scrunch5(x)
    assert m.size == 1000
    assert np.array_equal(m, np.median(x[:5000].reshape(-1, 5), axis=1))
    for k in (1, 2, 3, 4):
        v = oracle.median_scrunch5(x[:k])
        assert v.size == 1 and v[0] == np.median(x[:k])
    s = oracle.linear_stretch(np.array([0.0, 1.0, 4.0]), 5)
    assert np.allclose(s, [0.0, 0.5, 1.0, 2.5, 4.0])


def test_peak_clustering_rule(oracle):
    # a cluster continues while the next bin is < min_gap from the bin
    # holding the current maximum
    idx = np.array([10, 20, 35, 60, 100, 129, 158, 190])
    snr = np.array([8.0, 9.0, 7.5, 8.5, 9.5, 9.0, 9.6, 7.1])
    pi, ps = oracle.identify_unique_peaks(idx, snr, 30)
    # 10..35 cluster around 20; 60 alone; 100 absorbs 129 (29 < 30) but
    # not 158 (58 from the maximum at 100); 158 alone; 190 alone
    assert list(pi) == [20, 60, 100, 158, 190]
    assert list(ps) == [9.0, 8.5, 9.5, 9.6, 7.1]


def test_harmonic_sum_order_and_index(oracle):
    rng = np.random.default_rng(3)
    p = rng.standard_normal(4097)
    s = oracle.harmonic_sums(p, 5)
    i = 3000
    val = p[i]
    fr = [[(1, 2)], [(3, 4), (1, 4)], [(m, 8) for m in (1, 3, 5, 7)],
          [(m, 16) for m in range(1, 16, 2)], [(m, 32) for m in range(1, 32, 2)]]
    for h, terms in enumerate(fr, start=1):
        for m, d in terms:
            val += p[int(i * m / d + 0.5)]
        assert s[h - 1, i] == pytest.approx(val * 2.0 ** (-h / 2), rel=1e-15)
    with pytest.raises(ValueError):
        oracle.harmonic_sums(p, 6)


def test_search_recovers_injected_pulsar(oracle):
    from peasoup_b200 import synth
    n, ts = 1 << 17, 64e-6
    x = synth.make_series_np(synth.SeriesSpec(nsamps=n, tsamp=ts, sigma=1.0, pulsars=[
        synth.Pulsar(5.7e-3, 12.0, 0.05, 1.0)]), 0)
    p = oracle.SearchParams(fft_size=n, tsamp=ts, acc_lo=-50.0, acc_hi=50.0, nharmonics=4,
                            min_snr=7.0, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ)
    c, tr = oracle.search_dm(x, p)
    f0 = 1 / 5.7e-3
    best = c[np.argmax(c["snr"])]
    assert abs(best["freq"] - f0) < 2 * (1 / (n * ts))


# ------------------------------------------------------------ against the reference build
@pytest.fixture(scope="module")
def gi(rg):
    """The seeded inputs the reference ran on, regenerated and checked."""
    import sys
    sys.path.insert(0, GOLD)
    import golden_inputs as GI
    inp = GI.inputs()
    for k, v in inp.items():
        assert GI.sha(v) == str(rg[f"sha_{k}"]), f"input {k} does not regenerate"
    return GI, inp


def test_oracle_resample_index_matches_reference(oracle, rg, gi):
    GI, _ = gi
    for n in GI.RESAMPLE_SIZES:
        for nm, fn in (("resampleII", oracle.resampleII_index),):
            d = rg[f"{nm}_{n}_delta"].astype(np.int64)
            for t, a in enumerate(GI.RESAMPLE_ACCS):
                got = fn(n, float(a), float(GI.RESAMPLE_TSAMP)).astype(np.int64) - np.arange(n)
                assert np.array_equal(got, d[t]), (n, a, np.count_nonzero(got != d[t]))


def test_centred_resample_index_matches_reference(oracle, rg, gi):
    """The centred form's rounding depends on contraction; the reference's
    maps must equal one of the two evaluations for every acceleration."""
    GI, _ = gi
    for n in GI.RESAMPLE_SIZES:
        d = rg[f"resample_{n}_delta"].astype(np.int64)
        for t, a in enumerate(GI.RESAMPLE_ACCS):
            v = [oracle.resample_index(n, float(a), float(GI.RESAMPLE_TSAMP), f).astype(np.int64)
                 - np.arange(n) for f in (0, 1)]
            assert np.array_equal(v[0], d[t]) or np.array_equal(v[1], d[t]), (n, a)


def test_oracle_stages_match_reference(oracle, rg, gi):
    GI, inp = gi
    x = inp["fft_in"].astype(np.float64)
    assert err_vs_rms(oracle.rfft(x), rg["fft_r2c"]) < 1e-5
    assert err_vs_rms(oracle.irfft(inp["fft_c2r_in"].astype(np.complex128), 1 << 12),
                      rg["fft_c2r"]) < 1e-5
    X = inp["form_in"].astype(np.complex128)
    assert rel_err(oracle.form_power(X), rg["form_power"]) < 1e-6
    assert rel_err(oracle.form_interbin(X), rg["form_interbin"]) < 1e-6
    med = oracle.running_median(inp["median_in"].astype(np.float64), GI.MEDIAN_BW)
    assert rel_err(med, rg["median_out"]) < 1e-6
    Xd = oracle.deredden(inp["dered_X"].astype(np.complex128), med)
    assert err_vs_rms(Xd, rg["dered_out"]) < 1e-5
    Z = oracle.zap(inp["dered_X"].astype(np.complex128), float(np.float32(GI.MEDIAN_BW)),
                   GI.ZAP_FREQS, GI.ZAP_WIDTHS)
    assert np.array_equal(Z.astype(np.complex64), rg["zap_out"])
    m, r, sd = oracle.stats(inp["stats_in"].astype(np.float64))
    assert np.allclose([m, r, sd], rg["stats_out"], rtol=1e-6)
    nrm = oracle.normalise(inp["stats_in"].astype(np.float64), 1.25, 0.75)
    assert rel_err(nrm, rg["norm_out"]) < 1e-6
    base, _ = oracle.remove_baseline(inp["baseline_in"].astype(np.float64))
    assert err_vs_rms(base, rg["baseline_out"]) < 1e-4
    # FP32 accumulation of up to 32 terms in the reference: ~3e-6 of RMS
    hs = oracle.harmonic_sums(inp["harm_in"].astype(np.float64), 5)
    for h in range(5):
        assert err_vs_rms(hs[h], rg["harm_out"][h]) < 1e-5
    spec = inp["peaks_in"].astype(np.float64)
    for nh in range(6):
        _, sn, fr = oracle.find_peaks(spec, GI.MEDIAN_BW, nh, 7.0, 0.1, 1100.0)
        assert np.array_equal(fr, rg[f"peaks_{nh}_freq"]), nh
        assert np.allclose(sn, rg[f"peaks_{nh}_snr"], rtol=1e-6), nh


@pytest.mark.parametrize("case", ["w1", "w2"])
def test_oracle_worker_matches_reference(oracle, rg, gi, case):
    from peasoup_b200 import synth
    GI, _ = gi
    name, series, dms, ts, n, kw, zap = [c for c in GI.worker_cases() if c[0] == case][0]
    assert GI.sha(series) == str(rg[f"sha_{case}_series"])
    zf, zw = zap if zap is not None else (np.zeros(0, np.float32), np.zeros(0, np.float32))
    tobs = float(np.float32(np.float32(n) * np.float32(ts)))
    got = []
    for d in range(len(dms)):
        p = oracle.SearchParams(fft_size=n, tsamp=ts, dm=float(dms[d]), dm_idx=d,
                                cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ, birdie_freqs=zf,
                                birdie_widths=zw, **kw)
        c, _ = oracle.search_dm(series[d], p)
        surv, _, _, _ = oracle.accel_distill(c, tobs, 1e-4)
        got.append(surv)
    got = np.concatenate(got)
    nm, ua, ub, worst = match_candidates(got, rg[f"{case}_cands"], float(kw["min_snr"]))
    assert not ua and not ub, (ua[:5], ub[:5])
    assert nm > 0 and worst < 1e-3
