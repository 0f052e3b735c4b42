"""The per-DM acceleration search (the fused B200 path) and the worker loop
that drives it over a block of DM trials.

``AccelSearch`` owns one ``psx_search`` instance (device buffers, cuFFT
plans and captured schedules for one transform length) and runs the body
of the reference's DM loop (src/pipeline_multi.cu:161-294) per call.
``Worker`` mirrors the reference's Worker/DMDispenser pair
(pipeline_multi.cu:38-305): it pulls DM indices from a dispenser and
collects the per-DM candidate lists.
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import SearchConfig, SearchInfo, SearchProfile, check, load

CAND_DTYPE = np.dtype([("dm", "<f4"), ("dm_idx", "<i4"), ("acc", "<f4"),
                       ("nh", "<i4"), ("snr", "<f4"), ("freq", "<f4")])


@dataclass
class SearchParams:
    """The CmdLineOptions fields the Worker reads, with the reference's
    defaults (include/utils/cmdline.hpp:99-191)."""
    fft_size: int
    tsamp: float
    cdm: float = 0.0
    acc_lo: float = 0.0
    acc_hi: float = 0.0
    acc_tol: float = 1.10
    acc_pulse_width: float = 64e-6
    cfreq_hz: float = 1475.12e6
    ch_bw_hz: float = 1.09e6
    nharmonics: int = 4
    min_snr: float = 9.0
    min_freq: float = 0.1
    max_freq: float = 1100.0
    min_gap: int = 30
    freq_tol: float = 1e-4
    max_harm: float = 16.0
    boundary_5_freq: float = 0.05
    boundary_25_freq: float = 0.5
    birdie_freqs: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    birdie_widths: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    mode: str = "batched"          # "plain": one trial per launch
    batch: int = 0                 # 0: chosen from the transform length
    # resample inside cuFFT through an LTO load callback: refused
    # (PSX_ERR_UNSUPPORTED), since the cuFFT 11.4 library of CUDA 12.9 fails
    # plan creation for LTO callbacks on sm_100; the two-pass transform
    # (fft_form 3) gathers the resampled series in its first pass instead.
    fft_callback: bool = False
    graph: bool = True             # batched: CUDA-graph trial schedule
    harm_shape: int = 0            # harmonic-kernel tile shape (0 = default)
    lanes: int = 0                 # batched: streams the launch groups alternate over (0 = 1)
    fft_form: int = 0              # batched: 0 default (3 for 2^19..2^25, 3*2^17..3*2^23, else 1),
                                   # 1 cuFFT complex transform + fused unpack/interbin,
                                   # 2 the reference's real transform + interbin,
                                   # 3 the library's two-pass transform (resample in pass 1)
    group_dms: int = 0             # batched: DM trials whose prologues run as one batch
                                   # (0 default: 4 for <= 2^22 points and few trials
                                   # per DM trial; 1 off; 2..16 that many)

    def to_c(self):
        cfg = SearchConfig()
        load().psx_search_config_defaults(C.byref(cfg), self.fft_size, self.tsamp)
        for k in ("cdm", "acc_lo", "acc_hi", "acc_tol", "acc_pulse_width", "cfreq_hz",
                  "ch_bw_hz", "nharmonics", "min_snr", "min_freq", "max_freq", "min_gap",
                  "freq_tol", "max_harm", "boundary_5_freq", "boundary_25_freq", "batch"):
            setattr(cfg, k, getattr(self, k))
        bf = np.ascontiguousarray(self.birdie_freqs, np.float32)
        bw = np.ascontiguousarray(self.birdie_widths, np.float32)
        keep = (bf, bw)
        if bf.size:
            cfg.birdie_freqs = bf.ctypes.data_as(C.POINTER(C.c_float))
            cfg.birdie_widths = bw.ctypes.data_as(C.POINTER(C.c_float))
            cfg.nbirdies = bf.size
        cfg.mode = _lib.PSX_MODE_PLAIN if self.mode == "plain" else _lib.PSX_MODE_BATCHED
        cfg.use_fft_callback = int(self.fft_callback)
        cfg.use_graph = int(self.graph)
        cfg.harm_shape = int(self.harm_shape)
        cfg.lanes = int(self.lanes)
        cfg.fft_form = int(self.fft_form)
        cfg.group_dms = int(self.group_dms)
        return cfg, keep


def autotune(params: SearchParams, batches=(2, 4, 8, 16), reps: int = 2,
             max_trials: int = 128) -> dict:
    """Times every (trials per launch group, harmonic-kernel shape) pair on
    synthetic noise of params.fft_size samples (psx_autotune) and returns
    {"batch", "harm_shape", "ms_per_dm": {(batch, shape): ms}}; the choice
    changes grouping only, never results."""
    cfg, keep = params.to_c()
    b = np.ascontiguousarray(batches, np.int32)
    ms = np.zeros(len(b) * _lib.PSX_HARM_SHAPES, np.float64)
    check(load().psx_autotune(C.byref(cfg), b.ctypes.data_as(C.c_void_p), len(b), reps,
                              max_trials, ms.ctypes.data_as(C.c_void_p)), "autotune")
    del keep
    table = {(int(bb), sh + 1): float(ms[i * _lib.PSX_HARM_SHAPES + sh])
             for i, bb in enumerate(b) for sh in range(_lib.PSX_HARM_SHAPES)}
    return {"batch": int(cfg.batch), "harm_shape": int(cfg.harm_shape), "ms_per_dm": table}


def footprint(params: SearchParams) -> int:
    """Device bytes one AccelSearch for these parameters holds."""
    cfg, _keep = params.to_c()
    return int(load().psx_search_footprint(C.byref(cfg)))


class AccelSearch:
    """One search instance on the current CUDA device."""

    def __init__(self, params: SearchParams):
        self.params = params
        cfg, keep = params.to_c()
        self._handle = C.c_void_p()
        check(load().psx_search_create(C.byref(cfg), C.byref(self._handle)), "search_create")
        del keep
        self._cap = 1 << 16
        self._out = np.zeros(self._cap, CAND_DTYPE)
        self._na = np.zeros(self._cap, np.int32)
        self._tr = np.zeros(self._cap, np.int32)

    def close(self) -> None:
        if self._handle:
            load().psx_search_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int) -> None:
        check(load().psx_search_set_stream(self._handle, C.c_void_p(stream_handle)),
              "search_set_stream")

    def search(self, series, dm: float = 0.0, dm_idx: int = 0, per_dm: bool = True,
               nsamps: Optional[int] = None):
        """Search one dedispersed series (a host numpy array or a CUDA
        tensor).  Returns (candidates, nassoc, trial_index): with per_dm the
        reference Worker's acceleration-distilled list (dm_trial_cands),
        otherwise every trial's harmonic-distilled list in trial order."""
        on_dev = 0
        if hasattr(series, "is_cuda") and series.is_cuda:
            ptr = C.c_void_p(series.data_ptr())
            n = series.numel() if nsamps is None else nsamps
            on_dev = 1
            keep = series
        else:
            a = np.ascontiguousarray(series, np.float32)
            ptr = C.c_void_p(a.ctypes.data)
            n = a.size if nsamps is None else nsamps
            keep = a
        out_mode = (_lib.PSX_OUT_DM_FOREST if per_dm == "forest" else
                    _lib.PSX_OUT_DM if per_dm else _lib.PSX_OUT_TRIAL)
        nout = C.c_size_t()
        L = load()
        while True:
            rc = L.psx_search_dm(self._handle, ptr, n, on_dev, dm, dm_idx, out_mode,
                                 self._out.ctypes.data, self._na.ctypes.data,
                                 self._tr.ctypes.data, self._cap, C.byref(nout))
            if rc == _lib.PSX_ERR_OVERFLOW and nout.value > self._cap:
                self._cap = int(nout.value * 1.5) + 1024
                self._out = np.zeros(self._cap, CAND_DTYPE)
                self._na = np.zeros(self._cap, np.int32)
                self._tr = np.zeros(self._cap, np.int32)
                continue
            check(rc, "search_dm")
            break
        del keep
        k = nout.value
        return self._out[:k].copy(), self._na[:k].copy(), self._tr[:k].copy()

    def search_block(self, series, dms, dm_idx=None, per_dm=True):
        """Search a block of DM trials (a sequence of host arrays, a 2-D
        array, or a sequence / 2-D CUDA tensor), overlapping the host-side
        clustering of one DM with the GPU search of the next.  Returns
        (candidates, nassoc, trial_index, dm_position).  per_dm="forest"
        returns each DM's acceleration-distilled candidates with their
        association trees: a candidate forest whose subtree sizes take the
        place of nassoc (see peasoup_b200.output)."""
        rows = [series[i] for i in range(len(series))]
        n = len(rows)
        on_dev = int(hasattr(rows[0], "is_cuda") and rows[0].is_cuda)
        keep = []
        if on_dev:
            ptrs = (C.c_void_p * n)(*[r.data_ptr() for r in rows])
            nsamps = rows[0].numel()
        else:
            arrs = [np.ascontiguousarray(r, np.float32) for r in rows]
            keep = arrs
            ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
            nsamps = arrs[0].size
        dm_arr = np.ascontiguousarray(dms, np.float32)
        idx_arr = np.ascontiguousarray(np.arange(n) if dm_idx is None else dm_idx, np.int32)
        out_mode = (_lib.PSX_OUT_DM_FOREST if per_dm == "forest" else
                    _lib.PSX_OUT_DM if per_dm else _lib.PSX_OUT_TRIAL)
        nout = C.c_size_t()
        L = load()
        while True:
            dmpos = np.zeros(self._cap, np.int32)
            rc = L.psx_search_block(self._handle, ptrs, nsamps, on_dev, dm_arr.ctypes.data,
                                    idx_arr.ctypes.data, n, out_mode, self._out.ctypes.data,
                                    self._na.ctypes.data, self._tr.ctypes.data,
                                    dmpos.ctypes.data, self._cap, C.byref(nout))
            if rc == _lib.PSX_ERR_OVERFLOW and nout.value > self._cap:
                self._cap = int(nout.value * 1.5) + 1024
                self._out = np.zeros(self._cap, CAND_DTYPE)
                self._na = np.zeros(self._cap, np.int32)
                self._tr = np.zeros(self._cap, np.int32)
                continue
            check(rc, "search_block")
            break
        del keep
        k = nout.value
        return (self._out[:k].copy(), self._na[:k].copy(), self._tr[:k].copy(),
                dmpos[:k].copy())

    def set_profile(self, on: bool = True) -> None:
        """Record CUDA events around every launch group (stage timings)."""
        check(load().psx_search_set_profile(self._handle, int(on)), "search_set_profile")

    def profile(self, reset: bool = False) -> dict:
        p = SearchProfile()
        check(load().psx_search_get_profile(self._handle, C.byref(p), int(reset)),
              "search_get_profile")
        return {f: getattr(p, f) for f, _ in SearchProfile._fields_}

    def info(self) -> dict:
        i = SearchInfo()
        check(load().psx_search_last_info(self._handle, C.byref(i)), "search_last_info")
        return {f: getattr(i, f) for f, _ in SearchInfo._fields_}

    def debug_tap(self, trial: int):
        """Dereddened series, resampled series and normalised spectrum of
        trial `trial` of the last call, plus (mean*N, std*N)."""
        N = self.params.fft_size
        B = N // 2 + 1
        tim = np.zeros(N, np.float32)
        tr = np.zeros(N, np.float32)
        ps = np.zeros(B, np.float32)
        nm = np.zeros(2, np.float32)
        check(load().psx_search_debug_tap(self._handle, trial, tim.ctypes.data, tr.ctypes.data,
                                          ps.ctypes.data, nm.ctypes.data), "search_debug_tap")
        return tim, tr, ps, nm


class DMDispenser:
    """pipeline_multi.cu:38-86: hands out DM indices to workers."""

    def __init__(self, count: int):
        self.count = count
        self._next = 0
        self._lock = threading.Lock()

    def get_dm_trial_idx(self) -> int:
        with self._lock:
            if self._next >= self.count:
                return -1
            i = self._next
            self._next += 1
            return i


class Worker:
    """pipeline_multi.cu:88-305: searches DM trials pulled from a dispenser
    and collects the per-DM acceleration-distilled candidates."""

    def __init__(self, series_block, dms, params: SearchParams, dispenser: DMDispenser,
                 search: Optional[AccelSearch] = None):
        self.series = series_block
        self.dms = np.asarray(dms, np.float32)
        self.params = params
        self.dispenser = dispenser
        self.search = search or AccelSearch(params)
        self.dm_trial_cands: List[np.ndarray] = []
        self.nassoc: List[np.ndarray] = []

    def start(self) -> None:
        while True:
            ii = self.dispenser.get_dm_trial_idx()
            if ii == -1:
                break
            c, na, _ = self.search.search(self.series[ii], float(self.dms[ii]), ii, per_dm=True)
            self.dm_trial_cands.append(c)
            self.nassoc.append(na)

    def candidates(self) -> np.ndarray:
        if not self.dm_trial_cands:
            return np.zeros(0, CAND_DTYPE)
        return np.concatenate(self.dm_trial_cands)
