"""Writes ref_golden.npz: outputs of the reference's OWN CUDA implementation
(src/kernels.cu, include/transforms/*, the unmodified Worker of
src/pipeline_multi.cu, built for sm_100a into oracle/_ref by
oracle/Makefile) on small seeded inputs, for pinning the CPU oracle.

Needs a GPU and the built oracle/_ref/libpeasoup_ref_gpu.so:
    python tests/golden/make_ref_golden.py OUT.npz
Every input is stored next to the outputs it produced.
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from peasoup_b200 import synth  # noqa: E402

RESAMPLE_ACCS = np.array([-500.0, -123.4, -12.0, 12.0, 125.5, 500.0], np.float32)
RESAMPLE_TSAMP = np.float32(64e-6)


def search_case(name, g, series2d, dms, tsamp, fft_size, params: O.SearchParams, zap=None):
    zapfile = ""
    if zap is not None:
        fd, zapfile = tempfile.mkstemp(suffix=".txt")
        with os.fdopen(fd, "w") as f:
            for fr, w in zip(*zap):
                f.write(f"{fr:.3f} {w:.3f}\n")
    cands, na = O.ref_worker_search(series2d, tsamp, dms, fft_size, params, zapfile)
    if zapfile:
        os.unlink(zapfile)
        g[f"{name}_zap_freqs"] = np.asarray(zap[0], np.float32)
        g[f"{name}_zap_widths"] = np.asarray(zap[1], np.float32)
    g[f"{name}_series"] = np.asarray(series2d, np.float32)
    g[f"{name}_dms"] = np.asarray(dms, np.float32)
    g[f"{name}_meta"] = np.array([tsamp, fft_size, params.acc_lo, params.acc_hi,
                                  params.nharmonics, params.min_snr, params.cdm], np.float64)
    g[f"{name}_cands"] = cands
    g[f"{name}_nassoc"] = na


def main(out_path):
    O.ref_gpu()
    g = {}
    rng = np.random.default_rng(11)

    # resampler index maps: the input x[i] = i makes the output the index
    for n in (1 << 18, 3 << 16):
        x = np.arange(n, dtype=np.float32)
        for nm, fn in (("resampleII", O.ref_resampleII), ("resample", O.ref_resample)):
            d = np.stack([fn(x, float(a), float(RESAMPLE_TSAMP)).astype(np.int64) - np.arange(n)
                          for a in RESAMPLE_ACCS])
            g[f"{nm}_{n}_delta"] = d.astype(np.int32)
    g["resample_accs"] = RESAMPLE_ACCS
    g["resample_tsamp"] = np.float32(RESAMPLE_TSAMP)

    # FFTs
    x = rng.standard_normal(1 << 14).astype(np.float32)
    g["fft_in"] = x
    g["fft_r2c"] = O.ref_fft_r2c(x)
    X = (rng.standard_normal((1 << 13) + 1) + 1j * rng.standard_normal((1 << 13) + 1)).astype(np.complex64)
    X[0] = X[0].real
    X[-1] = X[-1].real
    g["fft_c2r_in"] = X
    g["fft_c2r"] = O.ref_fft_c2r(X, 1 << 14)

    # spectrum forming
    X = (rng.standard_normal((1 << 14) + 1) + 1j * rng.standard_normal((1 << 14) + 1)).astype(np.complex64)
    X[7] = 0
    g["form_in"] = X
    g["form_power"] = O.ref_form(X, False)
    g["form_interbin"] = O.ref_form(X, True)

    # running median and dereddening (a red-ish amplitude spectrum)
    nb = (1 << 16) + 1
    bw = float(np.float32(1.0 / np.float32(np.float32(1 << 17) * np.float32(64e-6))))
    amp = (np.abs(rng.standard_normal(nb) + 1j * rng.standard_normal(nb)) *
           (1 + 50.0 / (1 + np.arange(nb) / 40.0))).astype(np.float32)
    g["median_in"] = amp
    g["median_bw"] = np.float64(bw)
    g["median_out"] = O.ref_running_median(amp, bw)
    Xd = (rng.standard_normal(nb) + 1j * rng.standard_normal(nb)).astype(np.complex64)
    g["dered_X"] = Xd
    g["dered_out"] = O.ref_deredden(Xd, amp, bw)

    # zapping
    zf = np.array([0.3, 17.25, 50.0, 100.0, 1990.0, 5000.0], np.float32)
    zw = np.array([0.05, 0.1, 0.1, 0.15, 20.0, 1.0], np.float32)
    fd, zp = tempfile.mkstemp(suffix=".txt")
    with os.fdopen(fd, "w") as f:
        for a, b in zip(zf, zw):
            f.write(f"{a:.3f} {b:.3f}\n")
    g["zap_freqs"], g["zap_widths"] = zf, zw
    g["zap_out"] = O.ref_zap(Xd, bw, zp)
    os.unlink(zp)

    # statistics, normalisation, baseline removal
    p = np.abs(rng.standard_normal(nb)).astype(np.float32) * 3 + 1
    g["stats_in"] = p
    g["stats_out"] = np.array(O.ref_stats(p), np.float32)
    g["norm_out"] = O.ref_normalise(p, 1.25, 0.75)
    tim = (128 + 20 * rng.standard_normal(1 << 16)).astype(np.float32)
    g["baseline_in"] = tim
    g["baseline_out"] = O.ref_remove_baseline(tim)

    # harmonic sums
    s = rng.standard_normal((1 << 15) + 1).astype(np.float32)
    g["harm_in"] = s
    g["harm_out"] = O.ref_harmonic_sums(s, 5)

    # peak finding per harmonic number
    spec = rng.standard_normal((1 << 15) + 1).astype(np.float32)
    for c in (100, 101, 140, 175, 3000, 3020, 3051, 9000, 20000, 32700):
        spec[c] = 12.0 + (c % 7)
    spec[3010] = 13.5
    g["peaks_in"] = spec
    g["peaks_bw"] = np.float64(bw)
    for nh in range(6):
        sn, fr = O.ref_find_candidates(spec, bw, nh, 7.0, 0.1, 1100.0)
        g[f"peaks_{nh}_snr"], g[f"peaks_{nh}_freq"] = sn, fr

    # full Worker runs
    n1 = 1 << 17
    s1 = synth.make_series_np(synth.SeriesSpec(
        nsamps=n1, tsamp=64e-6, sigma=1.0,
        pulsars=[synth.Pulsar(period=5.7e-3, accel=12.0, duty=0.05, amp=1.0)]), 0)
    p1 = O.SearchParams(fft_size=n1, tsamp=64e-6, acc_lo=-50.0, acc_hi=50.0, nharmonics=4,
                        min_snr=7.0, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ)
    search_case("w1", g, s1[None, :], [0.0], 64e-6, n1, p1)
    # two DMs, 5 folds, red noise, quantised, birdies zapped, padded
    n2 = 1 << 16
    plan = synth.survey_plan(ndm=2, nsamps=n2 - 1000, tsamp=76e-6, seed=3, npulsars=2,
                             nbirdies=5)
    for ps in plan.pulsars:
        ps.amp = 40.0
    s2 = np.stack([synth.survey_series_np(plan, d, seed=3) for d in range(2)])
    p2 = O.SearchParams(fft_size=n2, tsamp=76e-6, acc_lo=-100.0, acc_hi=100.0, nharmonics=5,
                        min_snr=6.0, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ, cdm=0.0)
    search_case("w2", g, s2, plan.dms, 76e-6, n2, p2, zap=(plan.birdie_freqs, plan.birdie_widths))
    np.savez_compressed(out_path, **g)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden",
                                                            "ref_golden.npz"))
