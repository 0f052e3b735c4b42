"""Writes ref_golden.npz: outputs of the reference's OWN CUDA implementation
(src/kernels.cu, include/transforms/*, the unmodified Worker of
src/pipeline_multi.cu, built for sm_100a into oracle/_ref by
oracle/Makefile) on the seeded inputs of golden_inputs.py, for pinning the
CPU oracle.  Stores outputs plus the SHA-256 of every input.

Needs a GPU and oracle/_ref/libpeasoup_ref_gpu.so:
    python tests/golden/make_ref_golden.py OUT.npz
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import golden_inputs as GI  # noqa: E402
from oracle import oracle as O  # noqa: E402
from peasoup_b200 import synth  # noqa: E402


def main(out_path):
    O.ref_gpu()
    g = {}
    inp = GI.inputs()
    for k, v in inp.items():
        g[f"sha_{k}"] = np.array(GI.sha(v))
    # resampler index maps: the input x[i] = i makes the output the index;
    # stored as the (small) difference to i
    for n in GI.RESAMPLE_SIZES:
        x = np.arange(n, dtype=np.float32)
        for nm, fn in (("resampleII", O.ref_resampleII), ("resample", O.ref_resample)):
            d = np.stack([fn(x, float(a), float(GI.RESAMPLE_TSAMP)).astype(np.int64) - np.arange(n)
                          for a in GI.RESAMPLE_ACCS])
            assert np.abs(d).max() < 127
            g[f"{nm}_{n}_delta"] = d.astype(np.int8)
    g["fft_r2c"] = O.ref_fft_r2c(inp["fft_in"])
    g["fft_c2r"] = O.ref_fft_c2r(inp["fft_c2r_in"], 1 << 12)
    g["form_power"] = O.ref_form(inp["form_in"], False)
    g["form_interbin"] = O.ref_form(inp["form_in"], True)
    g["median_out"] = O.ref_running_median(inp["median_in"], GI.MEDIAN_BW)
    g["dered_out"] = O.ref_deredden(inp["dered_X"], inp["median_in"], GI.MEDIAN_BW)
    fd, zp = tempfile.mkstemp(suffix=".txt")
    with os.fdopen(fd, "w") as f:
        for a, b in zip(GI.ZAP_FREQS, GI.ZAP_WIDTHS):
            f.write(f"{a:.3f} {b:.3f}\n")
    g["zap_out"] = O.ref_zap(inp["dered_X"], GI.MEDIAN_BW, zp)
    os.unlink(zp)
    g["stats_out"] = np.array(O.ref_stats(inp["stats_in"]), np.float32)
    g["norm_out"] = O.ref_normalise(inp["stats_in"], 1.25, 0.75)
    g["baseline_out"] = O.ref_remove_baseline(inp["baseline_in"])
    g["harm_out"] = O.ref_harmonic_sums(inp["harm_in"], 5)
    for nh in range(6):
        sn, fr = O.ref_find_candidates(inp["peaks_in"], GI.MEDIAN_BW, nh, 7.0, 0.1, 1100.0)
        g[f"peaks_{nh}_snr"], g[f"peaks_{nh}_freq"] = sn, fr
    for name, series, dms, ts, n, kw, zap in GI.worker_cases():
        p = O.SearchParams(fft_size=n, tsamp=ts, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ, **kw)
        zapfile = ""
        if zap is not None:
            fd, zapfile = tempfile.mkstemp(suffix=".txt")
            with os.fdopen(fd, "w") as f:
                for fr, w in zip(*zap):
                    f.write(f"{fr:.3f} {w:.3f}\n")
        cands, na = O.ref_worker_search(series, ts, dms, n, p, zapfile)
        if zapfile:
            os.unlink(zapfile)
        g[f"sha_{name}_series"] = np.array(GI.sha(series))
        g[f"{name}_cands"] = cands
        g[f"{name}_nassoc"] = na
    np.savez_compressed(out_path, **g)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_golden.npz"))
