"""Seeded inputs of the reference fixtures (ref_golden.npz).

Shared by make_ref_golden.py (which ran the reference's own build on them)
and by the tests (which regenerate them and check the stored SHA-256 of
every input before comparing outputs)."""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

RESAMPLE_ACCS = np.array([-500.0, -123.4, -12.0, 12.0, 125.5, 500.0], np.float32)
RESAMPLE_TSAMP = np.float32(64e-6)
RESAMPLE_SIZES = (1 << 18, 3 << 16)
NB = (1 << 13) + 1                     # bins of the spectrum-stage fixtures
MEDIAN_BW = float(np.float32(1.0 / np.float32(np.float32(1 << 14) * np.float32(64e-6))))
ZAP_FREQS = np.array([0.3, 17.25, 50.0, 100.0, 990.0, 5000.0], np.float32)
ZAP_WIDTHS = np.array([0.05, 0.1, 0.1, 0.15, 20.0, 1.0], np.float32)
PEAK_BINS = (100, 101, 140, 175, 3000, 3020, 3051, 5000, 7000, 8100)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def inputs():
    rng = np.random.default_rng(11)
    g = {}
    g["fft_in"] = rng.standard_normal(1 << 12).astype(np.float32)
    X = (rng.standard_normal((1 << 11) + 1) + 1j * rng.standard_normal((1 << 11) + 1)).astype(np.complex64)
    X[0] = X[0].real
    X[-1] = X[-1].real
    g["fft_c2r_in"] = X
    X = (rng.standard_normal(NB) + 1j * rng.standard_normal(NB)).astype(np.complex64)
    X[7] = 0
    g["form_in"] = X
    g["median_in"] = (np.abs(rng.standard_normal(NB) + 1j * rng.standard_normal(NB)) *
                      (1 + 50.0 / (1 + np.arange(NB) / 40.0))).astype(np.float32)
    g["dered_X"] = (rng.standard_normal(NB) + 1j * rng.standard_normal(NB)).astype(np.complex64)
    g["stats_in"] = (np.abs(rng.standard_normal(NB)) * 3 + 1).astype(np.float32)
    g["baseline_in"] = (128 + 20 * rng.standard_normal(1 << 14)).astype(np.float32)
    g["harm_in"] = rng.standard_normal((1 << 12) + 1).astype(np.float32)
    spec = rng.standard_normal(NB).astype(np.float32)
    for c in PEAK_BINS:
        spec[c] = 12.0 + (c % 7)
    spec[3010] = 13.5
    g["peaks_in"] = spec
    return g


def worker_cases():
    """(name, series [ndm, nsamps], dms, tsamp, fft_size, kwargs, zap)"""
    from peasoup_b200 import synth
    n1 = 1 << 17
    s1 = synth.make_series_np(synth.SeriesSpec(
        nsamps=n1, tsamp=64e-6, sigma=1.0,
        pulsars=[synth.Pulsar(period=5.7e-3, accel=12.0, duty=0.05, amp=1.0)]), 0)
    k1 = dict(acc_lo=-50.0, acc_hi=50.0, nharmonics=4, min_snr=7.0, cdm=0.0)
    n2 = 1 << 16
    plan = synth.survey_plan(ndm=2, nsamps=n2 - 1000, tsamp=76e-6, seed=3, npulsars=2,
                             nbirdies=5)
    for ps in plan.pulsars:
        ps.amp = 40.0
    s2 = np.stack([synth.survey_series_np(plan, d, seed=3) for d in range(2)])
    k2 = dict(acc_lo=-100.0, acc_hi=100.0, nharmonics=5, min_snr=6.0, cdm=0.0)
    return [("w1", s1[None, :], np.array([0.0], np.float32), 64e-6, n1, k1, None),
            ("w2", s2, plan.dms, 76e-6, n2, k2, (plan.birdie_freqs, plan.birdie_widths))]
