"""Peasoup's main program on one GPU.

search_to_outputs: the search part on a block of dedispersed series the
caller passes (one row per DM trial, as the reference's DispersionTrials
holds it): the Workers' DM loop (src/pipeline_multi.cu:111-303, 523-535),
then the global distillation, scoring and output files (:547-587).

run: the whole program from a SIGPROC filterbank (:342-587): segment
reading, DM list, dedispersion into device memory, search and outputs.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
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


# ------------------------------------------------------------ whole program
@dataclass
class Options:
    """The reference's CmdLineOptions with its defaults
    (include/utils/cmdline.hpp:7-40, 80-250).  Float options are float32,
    as the reference holds them."""
    infilename: str
    outdir: str = "peasoup_results"
    killfilename: str = ""
    zapfilename: str = ""
    max_num_threads: int = 14
    limit: int = 1000
    size: int = 0
    dm_file: str = "none"
    cdm: float = 0.0
    dm_start: float = 0.0
    dm_end: float = 0.0
    dm_tol: float = 1.11
    dm_pulse_width: float = 64.0
    host_ram_limit_gb: float = 20.0
    dedisp_gulp: int = 1000000
    acc_start: float = 0.0
    acc_end: float = 0.0
    acc_tol: float = 1.10
    acc_pulse_width: float = 64.0
    boundary_5_freq: float = 0.05
    boundary_25_freq: float = 0.5
    nharmonics: int = 4
    npdmp: int = 0
    min_snr: float = 9.0
    min_freq: float = 0.1
    max_freq: float = 1100.0
    max_harm: int = 16
    freq_tol: float = 0.0001
    verbose: bool = False
    progress_bar: bool = False
    start_sample: int = 0
    nsamples: int = 0
    timeseries_dump_dir: str = ""
    no_search: bool = False

    def f32(self, name: str) -> np.float32:
        return np.float32(getattr(self, name))


def _header_section(h) -> Dict[str, object]:
    """header_parameters (include/utils/output_stats.hpp:46-80)."""
    items: Dict[str, object] = {"source_name": h.source_name.decode(errors="replace"),
                                "rawdatafile": h.rawdatafile.decode(errors="replace")}
    for k in ("az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "period", "fch1",
              "foff", "nchans", "telescope_id", "machine_id", "data_type", "ibeam", "nbeams",
              "nbits", "barycentric", "pulsarcentric", "nbins", "nsamples", "nifs", "npuls",
              "refdm"):
        items[k] = getattr(h, k)
    items["signed"] = int(h.signed_data)
    return items


def _search_section(o: Options) -> Dict[str, object]:
    """search_parameters (include/utils/output_stats.hpp:90-120)."""
    f = o.f32
    return {"infilename": o.infilename, "outdir": o.outdir, "killfilename": o.killfilename,
            "zapfilename": o.zapfilename, "max_num_threads": o.max_num_threads, "size": o.size,
            "dmfilename": o.dm_file, "cdm": "%.4f" % f("cdm"), "dm_start": f("dm_start"),
            "dm_end": f("dm_end"), "dm_tol": f("dm_tol"), "dm_pulse_width": f("dm_pulse_width"),
            "acc_start": f("acc_start"), "acc_end": f("acc_end"), "acc_tol": f("acc_tol"),
            "acc_pulse_width": f("acc_pulse_width"), "boundary_5_freq": f("boundary_5_freq"),
            "boundary_25_freq": f("boundary_25_freq"), "nharmonics": o.nharmonics,
            "npdmp": o.npdmp, "min_snr": f("min_snr"), "min_freq": f("min_freq"),
            "max_freq": f("max_freq"), "max_harm": o.max_harm, "freq_tol": f("freq_tol"),
            "verbose": int(o.verbose), "progress_bar": int(o.progress_bar)}


def run(opts: Options, *, devices=(0,), params_overrides: Optional[Dict[str, object]] = None):
    """The reference's main program (src/pipeline_multi.cu:342-587) on one
    GPU: read the filterbank segment, make or read the DM list, dedisperse
    each DM chunk into device memory, search it, then distil, score and
    write candidates.peasoup and overview.xml into opts.outdir.  Returns
    what output.finish returns plus a dict of stage wall times.

    With opts.timeseries_dump_dir every dedispersed series is also written
    there as <stem>_DM<dm>.dat / .inf (sigproc.write_timeseries), and with
    opts.no_search as well nothing is searched and None is returned.  (The
    reference stops after dumping its first DM chunk,
    src/pipeline_multi.cu:505-515; here every chunk is dumped.)"""
    import torch

    from .dedisperse import Dedisperser
    from .sigproc import SigprocFilterbank, prev_power_of_two, read_dm_file
    from .transforms import AccelerationPlan, Zapper

    timers = {"reading": 0.0, "dedispersion": 0.0, "searching": 0.0, "folding": 0.0}
    t_total = time.perf_counter()
    if opts.nsamples > 0 and opts.size > 0 and opts.nsamples > opts.size:
        raise ValueError("nsamples cannot be > fft size.")
    nsamples = opts.size if (opts.size > 0 and opts.nsamples == 0) else opts.nsamples

    t0 = time.perf_counter()
    fil = SigprocFilterbank(opts.infilename, opts.start_sample, nsamples)
    header = fil.get_header()
    timers["reading"] = time.perf_counter() - t0
    size = prev_power_of_two(fil.get_effective_nsamps()) if opts.size == 0 else opts.size
    fil.size = size

    tsamp = np.float32(fil.get_tsamp())
    cfreq_hz = float(np.float32(float(np.float32(fil.get_cfreq())) * 1e6))
    ch_bw_hz = float(np.float32(float(np.float32(fil.get_foff())) * 1e6))
    pw = float(np.float32(float(opts.f32("acc_pulse_width")) * 1e-6))
    params = SearchParams(fft_size=size, tsamp=float(tsamp), cdm=float(opts.f32("cdm")),
                          acc_lo=float(opts.f32("acc_start")), acc_hi=float(opts.f32("acc_end")),
                          acc_tol=float(opts.f32("acc_tol")), acc_pulse_width=pw,
                          cfreq_hz=cfreq_hz, ch_bw_hz=ch_bw_hz, nharmonics=opts.nharmonics,
                          min_snr=float(opts.f32("min_snr")), min_freq=float(opts.f32("min_freq")),
                          max_freq=float(opts.f32("max_freq")),
                          freq_tol=float(opts.f32("freq_tol")), max_harm=float(opts.max_harm),
                          boundary_5_freq=float(opts.f32("boundary_5_freq")),
                          boundary_25_freq=float(opts.f32("boundary_25_freq")))
    if opts.zapfilename:
        z = Zapper(opts.zapfilename)
        params.birdie_freqs, params.birdie_widths = z.birdies, z.widths
    for k, v in (params_overrides or {}).items():
        setattr(params, k, v)

    if opts.dm_file == "none":
        dd = Dedisperser(fil)
        dd.generate_dm_list(opts.dm_start, opts.dm_end, opts.dm_pulse_width, opts.dm_tol)
        full_dm_list = dd.get_dm_list()
        dd.close()
    else:
        full_dm_list = read_dm_file(opts.dm_file)

    nbytes = float(np.float32(opts.host_ram_limit_gb * 1e9))
    gulp_dms = int(nbytes / (fil.get_effective_nsamps() * 4))
    if gulp_dms == 0:
        raise RuntimeError("Insufficient RAM specified to allow for dedispersion")
    # the dedispersed chunk stays in device memory: a third of it at most
    free, _ = torch.cuda.mem_get_info()
    gulp_dms = max(1, min(gulp_dms, len(full_dm_list),
                          int(free / 3 // (fil.get_effective_nsamps() * 4))))

    forests = []
    eng = AccelSearch(params)
    for start in range(0, len(full_dm_list), gulp_dms):
        chunk = full_dm_list[start:start + gulp_dms]
        t0 = time.perf_counter()
        dd = Dedisperser(fil)
        if opts.killfilename:
            dd.set_killmask(opts.killfilename)
        dd.set_dm_list(chunk)
        gulp = fil.get_effective_nsamps() if opts.dedisp_gulp == -1 else opts.dedisp_gulp
        trials = dd.dedisperse(None, fil.get_start_sample(), fil.get_end_sample(), gulp)
        torch.cuda.synchronize()
        timers["dedispersion"] += time.perf_counter() - t0
        if opts.timeseries_dump_dir:
            import os
            from .sigproc import write_timeseries
            os.makedirs(opts.timeseries_dump_dir, exist_ok=True)
            stem = os.path.splitext(os.path.basename(opts.infilename))[0]
            host = trials.to_host()
            for ii, dm in enumerate(chunk):
                write_timeseries(opts.timeseries_dump_dir, stem, host[ii], dm, header)
            if opts.no_search:
                dd.close()
                continue
        t0 = time.perf_counter()
        # DM indices restart in every chunk, as the reference's DMDispenser's do
        nodes, sizes, _, _ = eng.search_block(trials.rows(), chunk,
                                              np.arange(len(chunk), dtype=np.int32),
                                              per_dm="forest")
        forests.append((nodes, sizes))
        timers["searching"] += time.perf_counter() - t0
        dd.close()
        del trials
    eng.close()
    if opts.timeseries_dump_dir and opts.no_search:
        return None

    acc_plan = AccelerationPlan(params.acc_lo, params.acc_hi, params.acc_tol, params.acc_pulse_width,
                                size, params.tsamp, params.cfreq_hz, params.ch_bw_hz)
    accs = acc_plan.generate_accel_list(params.cdm, params.cdm)
    foff = np.float32(fil.get_foff())
    bw = float(np.float32(abs(foff) * np.float32(fil.get_nchans())))
    sections = {"header_parameters": _header_section(header),
                "search_parameters": _search_section(opts),
                "segment_parameters": {"segment_start_sample": fil.get_start_sample(),
                                       "segment_nsamples": fil.get_effective_nsamps(),
                                       "segment_pepoch": fil.get_segment_pepoch()}}
    timers["total"] = time.perf_counter() - t_total
    res = output.finish(forests, opts.outdir, tsamp=float(tsamp), cfreq_mhz=fil.get_cfreq(),
                        foff_mhz=float(foff), bw_mhz=bw, freq_tol=params.freq_tol,
                        max_harm=params.max_harm, limit_count=opts.limit, dms=full_dm_list,
                        accs=accs, cdm=params.cdm, sections=sections, devices=list(devices),
                        timings=timers)
    return res + (timers,)
