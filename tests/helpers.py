"""Comparison helpers shared by the parity tests."""
import numpy as np


def _wide(x):
    x = np.asarray(x)
    return x.astype(np.complex128) if np.iscomplexobj(x) else x.astype(np.float64)


def rel_err(a, b, floor_frac=1e-3):
    """max |a-b| / max(|b|, floor) with the floor a fraction of the RMS of
    b, so that bins near zero are judged against the spectrum's scale."""
    a = _wide(a)
    b = _wide(b)
    scale = np.sqrt(np.mean(np.abs(b) ** 2)) if b.size else 1.0
    den = np.maximum(np.abs(b), floor_frac * scale + 1e-300)
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0


def err_vs_rms(a, b):
    """max |a-b| relative to the RMS of b."""
    a = _wide(a)
    b = _wide(b)
    scale = np.sqrt(np.mean(np.abs(b) ** 2)) if b.size else 1.0
    return float(np.max(np.abs(a - b)) / scale) if a.size else 0.0


def err_vs_mag_or_rms(a, b):
    """max |a-b| / (|b| + RMS of b): relative where the values are large
    (spectral peaks, whose own FP32 rounding sets the error there),
    relative to the RMS elsewhere."""
    a = _wide(a)
    b = _wide(b)
    if not a.size:
        return 0.0
    scale = np.sqrt(np.mean(np.abs(b) ** 2))
    return float(np.max(np.abs(a - b) / (np.abs(b) + scale)))


def cand_key(c):
    return (int(c["dm_idx"]), float(c["acc"]), int(c["nh"]), float(c["freq"]))


def match_candidates(a, b, thresh, snr_rtol=1e-3, margin=2e-3):
    """Compare two candidate lists (structured arrays with dm_idx, acc, nh,
    freq, snr).  Exact (dm_idx, acc, nh, freq) identity is required for
    every candidate whose S/N clears the threshold by more than `margin`
    (relative); S/N of matched pairs must agree within snr_rtol.  Returns
    (n_matched, unmatched_a, unmatched_b, worst_snr_rel)."""
    ka = {cand_key(c): float(c["snr"]) for c in a}
    kb = {cand_key(c): float(c["snr"]) for c in b}
    matched = set(ka) & set(kb)
    worst = 0.0
    for k in matched:
        worst = max(worst, abs(ka[k] - kb[k]) / max(abs(kb[k]), 1e-30))
    ua = [(k, s) for k, s in ka.items() if k not in kb and s > thresh * (1 + margin)]
    ub = [(k, s) for k, s in kb.items() if k not in ka and s > thresh * (1 + margin)]
    return len(matched), ua, ub, worst
