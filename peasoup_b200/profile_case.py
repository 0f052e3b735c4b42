"""A small, self-contained search case for profiler captures.

    python -m peasoup_b200.profile_case [--ndm 2] [--nsamps 8388608] [--graph]
    python -m peasoup_b200.profile_case --dedisp [--ndm 32] [--nsamps 8388608]

Searches `ndm` DM trials of the survey-shape synthetic block (2^23
samples, tsamp 76 us, acceleration -100..100 m/s^2, 5 folds, 20 birdies)
with the batched engine and prints, per DM trial, the candidate count and
the engine's counters, then the per-stage CUDA-event profile.  Two DM
trials hold about 1.5 GB on the device (series, trial buffers, cuFFT work
area), so a capture of any of its kernels stays small while every buffer
a kernel streams exceeds the 126 MB L2.  Graph capture is off unless
`--graph` is given, so each kernel is an ordinary stream launch.

With --dedisp: `ndm` DM trials (DM_i = 0.5 i) of nsamps x nchans nbits-bit
rows (tsamp as given, a 70 MHz band from 1510 MHz down: foff -1.09 MHz at
64 channels), dedispersed four times from device memory; at 2^23 samples,
64 channels and 32 DM trials the case holds about 2.2 GB.
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
    ap.add_argument("--dedisp", action="store_true")
    ap.add_argument("--nchans", type=int, default=64)
    ap.add_argument("--nbits", type=int, default=8)
    a = ap.parse_args(argv)
    if a.dedisp:
        return dedisp_case(a)

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



def dedisp_case(a) -> int:
    import ctypes as C

    import numpy as np
    import torch
    from . import _lib, synth
    L = _lib.load()
    dms = (0.5 * np.arange(a.ndm)).astype(np.float32)
    plan = C.c_void_p()
    foff = synth.FOFF_MHZ * 64 / a.nchans
    _lib.check(L.psx_dedisp_create(a.nchans, a.tsamp, synth.FCH1_MHZ, foff, C.byref(plan)),
               "dedisp_create")
    _lib.check(L.psx_dedisp_set_dm_list(plan, dms.ctypes.data, dms.size), "set_dm_list")
    nout = a.nsamps - int(L.psx_dedisp_get_max_delay(plan))
    pitch = (nout + 3) // 4 * 4
    g = torch.Generator(device="cuda").manual_seed(7)
    rows = torch.randint(0, 256, (a.nsamps, a.nchans * a.nbits // 8), dtype=torch.uint8,
                         device="cuda", generator=g)
    out = torch.empty((a.ndm, pitch), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    for i in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        _lib.check(L.psx_dedisp_execute(plan, a.nsamps, C.c_void_p(rows.data_ptr()), a.nbits,
                                        C.c_void_p(out.data_ptr()), pitch, 0,
                                        C.c_void_p(st.cuda_stream)), "dedisp_execute")
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        print(f"dedisperse {a.ndm} DM x {nout} samples x {a.nchans} {a.nbits}-bit channels: "
              f"{ms:.3f} ms, "
              f"{a.ndm * nout * a.nchans / ms / 1e9:.3f} T channel-adds/s")
    L.psx_dedisp_destroy(plan)
    return 0


if __name__ == "__main__":
    sys.exit(main())
