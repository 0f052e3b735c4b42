"""The search part of peasoup's main program on a block of dedispersed
series: the Workers' DM loop (src/pipeline_multi.cu:111-303, 523-535) on
one GPU, then the global distillation, scoring and output files
(:547-587).  Reading the filterbank and dedispersing are not part of this
library; the caller passes the dedispersed block (one row per DM trial, as
the reference's DispersionTrials holds it) and the values the output
sections need.
"""
from __future__ import annotations

import time
from typing import Dict, Optional

import numpy as np

from . import output
from .search import AccelSearch, SearchParams


def search_to_outputs(block, dms, params: SearchParams, outdir: str, *, foff_mhz: float,
                      nchans: int, cfreq_mhz: Optional[float] = None, limit: int = 1000,
                      dm_chunk: int = 32, sections: Optional[Dict[str, Dict[str, object]]] = None,
                      devices=None):
    """Searches every row of `block` (host array or CUDA tensor) and writes
    candidates.peasoup and overview.xml into `outdir`.  The scorer's band is
    the reference's: centre frequency (MHz, default params.cfreq_hz) and
    |foff| * nchans (src/pipeline_multi.cu:550-552).  Returns what
    output.finish returns plus the per-stage wall times."""
    t0 = time.perf_counter()
    dms = np.ascontiguousarray(dms, np.float32)
    eng = AccelSearch(params)
    forests = []
    for c0 in range(0, len(dms), dm_chunk):
        idx = np.arange(c0, min(len(dms), c0 + dm_chunk), dtype=np.int32)
        nodes, sizes, _, _ = eng.search_block([block[i] for i in idx], dms[idx], idx,
                                              per_dm="forest")
        forests.append((nodes, sizes))
    eng.close()
    t1 = time.perf_counter()
    from .transforms import AccelerationPlan
    accs = AccelerationPlan(params.acc_lo, params.acc_hi, params.acc_tol, params.acc_pulse_width,
                            params.fft_size, params.tsamp, params.cfreq_hz,
                            params.ch_bw_hz).generate_accel_list(params.cdm, params.cdm)
    cf = params.cfreq_hz / 1e6 if cfreq_mhz is None else cfreq_mhz
    res = output.finish(forests, outdir, tsamp=params.tsamp, cfreq_mhz=cf, foff_mhz=foff_mhz,
                        bw_mhz=abs(foff_mhz) * nchans, freq_tol=params.freq_tol,
                        max_harm=params.max_harm, limit_count=limit, dms=dms, accs=accs,
                        cdm=params.cdm, sections=sections, devices=devices,
                        timings={"searching": t1 - t0})
    return res + ({"searching": t1 - t0, "total": time.perf_counter() - t0},)
