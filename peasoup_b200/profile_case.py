"""A small, self-contained search case for profiler captures.

    python -m peasoup_b200.profile_case [--ndm 2] [--nsamps 8388608] [--graph]

Searches `ndm` DM trials of the survey-shape synthetic block (2^23
samples, tsamp 76 us, acceleration -100..100 m/s^2, 5 folds, 20 birdies)
with the batched engine and prints, per DM trial, the candidate count and
the engine's counters, then the per-stage CUDA-event profile.  Two DM
trials hold about 1.5 GB on the device (series, trial buffers, cuFFT work
area), so a capture of any of its kernels stays small while every buffer
a kernel streams exceeds the 126 MB L2.  Graph capture is off unless
`--graph` is given, so each kernel is an ordinary stream launch.
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ndm", type=int, default=2)
    ap.add_argument("--nsamps", type=int, default=1 << 23)
    ap.add_argument("--tsamp", type=float, default=76e-6)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--graph", action="store_true")
    ap.add_argument("--harm-shape", type=int, default=0)
    a = ap.parse_args(argv)

    import torch
    from . import search, synth
    plan = synth.survey_plan(ndm=a.ndm, nsamps=a.nsamps, tsamp=a.tsamp)
    block = synth.survey_block_torch(plan)
    p = search.SearchParams(fft_size=a.nsamps, tsamp=a.tsamp, acc_lo=-100.0, acc_hi=100.0,
                            nharmonics=5, cfreq_hz=synth.CFREQ_HZ, ch_bw_hz=synth.CH_BW_HZ,
                            birdie_freqs=plan.birdie_freqs, birdie_widths=plan.birdie_widths,
                            batch=a.batch, graph=a.graph, harm_shape=a.harm_shape)
    s = search.AccelSearch(p)
    s.set_profile(not a.graph)
    for d in range(a.ndm):
        cands = s.search(block[d], float(plan.dms[d]), d)[0]
        print(d, len(cands), s.info(), flush=True)
    torch.cuda.synchronize()
    if not a.graph:
        print(s.profile(), flush=True)
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
