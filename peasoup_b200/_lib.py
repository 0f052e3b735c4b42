"""ctypes binding of libpeasoup_b200.so (the C ABI in include/peasoup_b200.h).

The library is built in-tree by peasoup_b200.build; loading fails loudly if
it is missing -- there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpeasoup_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "peasoup_b200.h")

PSX_OK = 0
PSX_ERR_INVALID = 1
PSX_ERR_CUDA = 2
PSX_ERR_CUFFT = 3
PSX_ERR_ALLOC = 4
PSX_ERR_OVERFLOW = 5
PSX_ERR_UNSUPPORTED = 6
PSX_ERR_IO = 7
PSX_ERR_BUSY = 8

PSX_FFT_R2C = 0
PSX_FFT_C2R = 1
PSX_FFT_C2C = 2
PSX_HARM_SHAPES = 7
PSX_MODE_PLAIN = 0
PSX_MODE_BATCHED = 1
PSX_OUT_TRIAL = 0
PSX_OUT_DM = 1
PSX_OUT_DM_FOREST = 2
PSX_DISTILL_HARMONIC = 0
PSX_DISTILL_ACCEL = 1
PSX_DISTILL_DM = 2
PSX_SERVE_LEAST_WORK = 0
PSX_SERVE_EVEN = 1
PSX_SERVE_EXCLUSIVE = 2


class PsxError(RuntimeError):
    """A failed library call (the reference raised std::runtime_error)."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


class Candidate(C.Structure):
    """psx_candidate == the reference's CandidatePOD (candidates.hpp:10-17)."""
    _fields_ = [("dm", C.c_float), ("dm_idx", C.c_int), ("acc", C.c_float),
                ("nh", C.c_int), ("snr", C.c_float), ("freq", C.c_float)]


class SearchConfig(C.Structure):
    _fields_ = [("fft_size", C.c_size_t), ("tsamp", C.c_float), ("cdm", C.c_float),
                ("acc_lo", C.c_float), ("acc_hi", C.c_float), ("acc_tol", C.c_float),
                ("acc_pulse_width", C.c_float), ("cfreq_hz", C.c_float),
                ("ch_bw_hz", C.c_float), ("nharmonics", C.c_int), ("min_snr", C.c_float),
                ("min_freq", C.c_float), ("max_freq", C.c_float), ("min_gap", C.c_int),
                ("freq_tol", C.c_float), ("max_harm", C.c_float),
                ("boundary_5_freq", C.c_float), ("boundary_25_freq", C.c_float),
                ("birdie_freqs", C.POINTER(C.c_float)), ("birdie_widths", C.POINTER(C.c_float)),
                ("nbirdies", C.c_size_t), ("mode", C.c_int), ("batch", C.c_int),
                ("use_fft_callback", C.c_int), ("use_graph", C.c_int), ("harm_shape", C.c_int),
                ("lanes", C.c_int), ("fft_form", C.c_int), ("group_dms", C.c_int)]


class SearchInfo(C.Structure):
    _fields_ = [("ntrials", C.c_int), ("nbatches", C.c_int), ("kernel_launches", C.c_int),
                ("fft_launches", C.c_int), ("above_threshold", C.c_longlong),
                ("fft_callback", C.c_int), ("graph", C.c_int), ("batch", C.c_int),
                ("baseline_passes", C.c_int), ("harm_shape", C.c_int),
                ("capture_fallbacks", C.c_int), ("fft_form", C.c_int),
                ("group_dms", C.c_int)]


class SearchProfile(C.Structure):
    _fields_ = [("prologue_ms", C.c_double), ("resample_ms", C.c_double),
                ("fft_ms", C.c_double), ("form_ms", C.c_double), ("harm_ms", C.c_double),
                ("groups", C.c_longlong), ("trials", C.c_longlong), ("dms", C.c_longlong),
                ("event_errors", C.c_longlong), ("last_event_error", C.c_int),
                ("host_enqueue_ms", C.c_double), ("host_wait_ms", C.c_double),
                ("host_collect_ms", C.c_double)]


class CandidateScore(C.Structure):
    _fields_ = [("is_physical", C.c_int), ("is_adjacent", C.c_int),
                ("ddm_count_ratio", C.c_float), ("ddm_snr_ratio", C.c_float),
                ("nassoc", C.c_int)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget", C.c_size_t), ("max_active", C.c_int),
                ("max_queue", C.c_int), ("policy", C.c_int)]


class RequestStats(C.Structure):
    _fields_ = [("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("footprint", C.c_size_t), ("ntrials", C.c_longlong), ("ndm", C.c_int),
                ("status", C.c_int), ("engine_reused", C.c_int)]


class SigprocHeader(C.Structure):
    """psx_sigproc_header == the keywords of SigprocHeader (header.hpp:171-212)."""
    _fields_ = [("source_name", C.c_char * 80), ("rawdatafile", C.c_char * 80),
                ("az_start", C.c_double), ("za_start", C.c_double), ("src_raj", C.c_double),
                ("src_dej", C.c_double), ("tstart", C.c_double), ("tsamp", C.c_double),
                ("period", C.c_double), ("fch1", C.c_double), ("foff", C.c_double),
                ("refdm", C.c_double), ("nchans", C.c_int), ("telescope_id", C.c_int),
                ("machine_id", C.c_int), ("data_type", C.c_int), ("ibeam", C.c_int),
                ("nbeams", C.c_int), ("nbits", C.c_int), ("barycentric", C.c_int),
                ("pulsarcentric", C.c_int), ("nbins", C.c_int), ("nsamples", C.c_int),
                ("nifs", C.c_int), ("npuls", C.c_int), ("signed_data", C.c_ubyte),
                ("header_size", C.c_size_t)]


PSX_DEDISP_RAW = 1

_vp = C.c_void_p
_sz = C.c_size_t
_f = C.c_float
_i = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "psx_last_error": (C.c_char_p, []),
    "psx_status_string": (C.c_char_p, [_i]),
    "psx_version": (C.c_char_p, []),
    "psx_resampleII": (_i, [_vp, _vp, _sz, _f, _f, _vp]),
    "psx_resample": (_i, [_vp, _vp, _sz, _f, _f, _vp]),
    "psx_resampleII_batch": (_i, [_vp, _vp, _sz, _vp, _i, _f, _vp]),
    "psx_form_power_series": (_i, [_vp, _vp, _sz, _i, _vp]),
    "psx_median_scrunch5": (_i, [_vp, _sz, _vp, _vp]),
    "psx_linear_stretch": (_i, [_vp, _sz, _vp, _sz, _vp]),
    "psx_running_median_scratch_bytes": (_sz, [_sz]),
    "psx_running_median": (_i, [_vp, _sz, C.c_double, _f, _f, _vp, _vp, _vp]),
    "psx_divide_c_by_f": (_i, [_vp, _vp, _sz, _vp]),
    "psx_deredden": (_i, [_vp, _vp, _sz, C.c_double, _f, _f, _vp, _vp]),
    "psx_zap_birdies": (_i, [_vp, _vp, _vp, _f, _sz, _sz, _vp]),
    "psx_read_zaplist": (_i, [C.c_char_p, _vp, _vp, _sz, C.POINTER(_sz)]),
    "psx_stats": (_i, [_vp, _sz, _sz, C.POINTER(_f), C.POINTER(_f), C.POINTER(_f), _vp]),
    "psx_normalise": (_i, [_vp, _f, _f, _sz, _vp]),
    "psx_remove_baseline": (_i, [_vp, _sz, C.POINTER(_i), _vp]),
    "psx_fill": (_i, [_vp, _sz, _f, _vp]),
    "psx_convert_u8_f32": (_i, [_vp, _vp, _sz, _vp]),
    "psx_convert_i8_f32": (_i, [_vp, _vp, _sz, _vp]),
    "psx_harmonic_sum": (_i, [_vp, _vp, _sz, _i, _vp]),
    "psx_find_peaks": (_i, [_vp, _i, _i, _f, _vp, _vp, _i, C.POINTER(_i), _vp]),
    "psx_find_peaks_noalloc": (_i, [_vp, _i, _i, _f, _vp, _vp, _i, C.POINTER(_i), _vp]),
    "psx_harmonic_peaks": (_i, [_vp, _sz, _sz, _i, _i, _vp, _vp, _f, _vp, _sz, C.POINTER(_sz),
                                C.c_uint, C.c_uint, _vp]),
    "psx_fft_plan_create": (_i, [C.POINTER(_vp), _sz, C.c_longlong, _i]),
    "psx_fft_exec": (_i, [_vp, _vp, _vp, _vp]),
    "psx_fft_exec_c2c": (_i, [_vp, _vp, _vp, _i, _vp]),
    "psx_fft_plan_destroy": (_i, [_vp]),
    "psx_accel_list": (_i, [_f, _f, _f, _f, _sz, _f, _f, _f, _f, _f, _vp, _sz, C.POINTER(_sz)]),
    "psx_peak_range": (_i, [C.c_uint, C.c_double, _i, _f, _f, C.POINTER(_i), C.POINTER(_i),
                            C.POINTER(_f)]),
    "psx_identify_unique_peaks": (_sz, [_vp, _vp, _sz, _i, _vp, _vp]),
    "psx_distill": (_sz, [_i, _vp, _sz, _f, _f, _f, _i, _i, _vp]),
    "psx_search_config_defaults": (None, [C.POINTER(SearchConfig), _sz, _f]),
    "psx_search_footprint": (_sz, [C.POINTER(SearchConfig)]),
    "psx_search_create": (_i, [C.POINTER(SearchConfig), C.POINTER(_vp)]),
    "psx_search_destroy": (_i, [_vp]),
    "psx_search_set_stream": (_i, [_vp, _vp]),
    "psx_search_dm": (_i, [_vp, _vp, _sz, _i, _f, _i, _i, _vp, _vp, _vp, _sz, C.POINTER(_sz)]),
    "psx_search_block": (_i, [_vp, _vp, _sz, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _sz,
                              C.POINTER(_sz)]),
    "psx_search_last_info": (_i, [_vp, C.POINTER(SearchInfo)]),
    "psx_search_set_profile": (_i, [_vp, _i]),
    "psx_search_set_priority": (_i, [_vp, _i]),
    "psx_search_get_profile": (_i, [_vp, C.POINTER(SearchProfile), _i]),
    "psx_search_debug_tap": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "psx_autotune": (_i, [C.POINTER(SearchConfig), _vp, _i, _i, _i, _vp]),
    "psx_search_retarget": (_i, [_vp, C.POINTER(SearchConfig)]),
    "psx_distill_forest": (_i, [_i, _vp, _vp, _sz, _f, _f, _f, _i, _i, _vp, _vp, _sz,
                                C.POINTER(_sz), C.POINTER(_sz)]),
    "psx_score_forest": (_i, [_vp, _vp, _sz, _f, _f, _f, _f, _vp, _sz, C.POINTER(_sz)]),
    "psx_write_candidates": (_i, [C.c_char_p, _vp, _vp, _sz, _vp, _sz, C.POINTER(_sz)]),
    "psx_overview_create": (_i, [C.POINTER(_vp)]),
    "psx_overview_destroy": (None, [_vp]),
    "psx_overview_add_section": (_i, [_vp, C.c_char_p, _vp, _vp, _sz]),
    "psx_overview_add_misc_info": (_i, [_vp, C.c_longlong]),
    "psx_overview_add_dm_list": (_i, [_vp, _vp, _sz]),
    "psx_overview_add_acc_list": (_i, [_vp, _vp, _sz, _f]),
    "psx_overview_add_device_info": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _sz]),
    "psx_overview_add_candidates": (_i, [_vp, _vp, _vp, _sz, _vp, _vp]),
    "psx_overview_write": (_i, [_vp, C.c_char_p, _vp, _sz, C.POINTER(_sz)]),
    "psx_server_create": (_i, [C.POINTER(ServerConfig), C.POINTER(_vp)]),
    "psx_server_destroy": (_i, [_vp]),
    "psx_server_clock": (C.c_double, [_vp]),
    "psx_server_submit": (_i, [_vp, C.POINTER(SearchConfig), _vp, _sz, _i, _vp, _vp, _i,
                               C.POINTER(C.c_longlong)]),
    "psx_server_wait": (_i, [_vp, C.c_longlong, C.c_double, _vp, _vp, _vp, _sz, C.POINTER(_sz),
                             C.POINTER(RequestStats)]),
    "psx_server_status": (_i, [_vp, C.POINTER(_sz), C.POINTER(_i), C.POINTER(_i),
                               C.POINTER(_i)]),
    "psx_sigproc_read_header": (_i, [C.c_char_p, C.POINTER(SigprocHeader)]),
    "psx_sigproc_parse_header": (_i, [_vp, _sz, C.POINTER(SigprocHeader)]),
    "psx_sigproc_read": (_i, [C.c_char_p, C.POINTER(SigprocHeader), _sz, _sz, _vp,
                              C.POINTER(_sz)]),
    "psx_sigproc_write_header": (_i, [C.c_char_p, C.POINTER(SigprocHeader), C.POINTER(_sz)]),
    "psx_read_dm_file": (_i, [C.c_char_p, _vp, _sz, C.POINTER(_sz)]),
    "psx_dedisp_create": (_i, [_sz, _f, _f, _f, C.POINTER(_vp)]),
    "psx_dedisp_destroy": (_i, [_vp]),
    "psx_dedisp_set_dm_list": (_i, [_vp, _vp, _sz]),
    "psx_dedisp_generate_dm_list": (_i, [_vp, _f, _f, _f, _f]),
    "psx_dedisp_get_dm_count": (_sz, [_vp]),
    "psx_dedisp_get_dm_list": (_i, [_vp, _vp, _sz]),
    "psx_dedisp_get_delay_table": (_i, [_vp, _vp]),
    "psx_dedisp_set_killmask": (_i, [_vp, _vp]),
    "psx_dedisp_get_max_delay": (_sz, [_vp]),
    "psx_dedisp_set_scratch_limit": (_i, [_vp, _sz]),
    "psx_dedisp_execute": (_i, [_vp, _sz, _vp, _i, _vp, _sz, _i, _vp]),
    "psx_dedisp_execute_host": (_i, [_vp, _sz, _vp, _i, _vp, _sz, _i, _vp]),
}

_lib = None


def declared_symbols() -> list:
    """Every function the public header declares."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(psx_[A-Za-z0-9_]+)\s*\(", txt)))


def load():
    """Load the in-tree library (never a copy elsewhere)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m peasoup_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return load().psx_last_error().decode(errors="replace")


def check(status: int, where: str) -> None:
    if status != PSX_OK:
        raise PsxError(status, where, last_error() or
                       load().psx_status_string(status).decode())
