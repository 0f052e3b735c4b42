"""ctypes bindings for the FP64 CPU oracle (``oracle/_build/liboracle.so``)
and for the reference's own implementation built in ``oracle/_ref``.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke``
and by the CPU-baseline leg of ``bench.py``.  The product never imports it.

The oracle restates, in double precision, the stages of Peasoup's per-DM
acceleration search (reference: src/kernels.cu, include/transforms/*.hpp,
src/pipeline_multi.cu:111-303).  See psx_oracle.h for the precision rule.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_HOST_PATH = os.path.join(HERE, "_ref", "libpeasoup_ref_host.so")
REF_GPU_PATH = os.path.join(HERE, "_ref", "libpeasoup_ref_gpu.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")

CAND_DTYPE = np.dtype([("dm", "<f4"), ("dm_idx", "<i4"), ("acc", "<f4"),
                       ("nh", "<i4"), ("snr", "<f4"), ("freq", "<f4")])


class _Cand(C.Structure):
    _fields_ = [("dm", C.c_float), ("dm_idx", C.c_int), ("acc", C.c_float),
                ("nh", C.c_int), ("snr", C.c_float), ("freq", C.c_float)]


class _Params(C.Structure):
    _fields_ = [("fft_size", C.c_size_t), ("tsamp", C.c_float),
                ("dm", C.c_float), ("cdm", C.c_float), ("dm_idx", C.c_int),
                ("acc_lo", C.c_float), ("acc_hi", C.c_float),
                ("acc_tol", C.c_float), ("acc_pulse_width", C.c_float),
                ("cfreq", C.c_float), ("ch_bw", C.c_float),
                ("nharmonics", C.c_int), ("min_snr", C.c_float),
                ("min_freq", C.c_float), ("max_freq", C.c_float),
                ("min_gap", C.c_int), ("freq_tol", C.c_float),
                ("max_harm", C.c_float),
                ("birdie_freqs", C.POINTER(C.c_float)),
                ("birdie_widths", C.POINTER(C.c_float)),
                ("nbirdies", C.c_size_t), ("resample_fused", C.c_int)]


class _Taps(C.Structure):
    _fields_ = [("tap_trial", C.c_int), ("tim_dered", C.POINTER(C.c_double)),
                ("tim_r", C.POINTER(C.c_double)), ("pspec", C.POINTER(C.c_double)),
                ("sums", C.POINTER(C.c_double)), ("median", C.POINTER(C.c_double)),
                ("stats", C.c_double * 3)]


def build() -> None:
    """Compile the oracle with gcc (a second or two)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def build_reference(ref_root: str = "/root/reference") -> bool:
    """Compile the reference's own implementation into oracle/_ref when its
    sources are present.  Returns True when both libraries exist."""
    if os.path.isdir(ref_root):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"], check=True)
    return os.path.exists(REF_HOST_PATH) and os.path.exists(REF_GPU_PATH)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_rfft.argtypes = [_dp, C.c_size_t, _dp]
        L.orc_irfft.argtypes = [_dp, C.c_size_t, _dp]
        L.orc_accel_fact.restype = C.c_double
        L.orc_accel_fact.argtypes = [C.c_float, C.c_float]
        L.orc_resampleII_index.argtypes = [C.c_size_t, C.c_float, C.c_float, C.c_int, _up]
        L.orc_resample_index.argtypes = [C.c_size_t, C.c_float, C.c_float, C.c_int, _up]
        L.orc_form_power.argtypes = [_dp, C.c_size_t, _dp]
        L.orc_form_interbin.argtypes = [_dp, C.c_size_t, _dp]
        L.orc_median_scrunch5.restype = C.c_size_t
        L.orc_median_scrunch5.argtypes = [_dp, C.c_size_t, _dp]
        L.orc_linear_stretch.argtypes = [_dp, C.c_size_t, _dp, C.c_size_t]
        L.orc_stretch_overreads.restype = C.c_size_t
        L.orc_splice_points.argtypes = [C.c_size_t, C.c_double, C.c_float, C.c_float,
                                        C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_running_median.argtypes = [_dp, C.c_size_t, C.c_double, C.c_float,
                                         C.c_float, _dp]
        L.orc_deredden.argtypes = [_dp, _dp, C.c_size_t]
        L.orc_zap_range.argtypes = [C.c_float, C.c_float, C.c_float, C.c_uint,
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_zap.argtypes = [_dp, C.c_size_t, C.c_float, _fp, _fp, C.c_size_t]
        L.orc_stats.argtypes = [_dp, C.c_size_t, C.c_size_t, C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_normalise.argtypes = [_dp, C.c_size_t, C.c_double, C.c_double]
        L.orc_remove_baseline.argtypes = [_dp, C.c_size_t]
        L.orc_harmonic_sums.argtypes = [_dp, C.c_size_t, C.c_int, _dp]
        L.orc_peak_range.argtypes = [C.c_uint, C.c_double, C.c_int, C.c_float, C.c_float,
                                     C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_float)]
        L.orc_identify_unique_peaks.restype = C.c_size_t
        L.orc_identify_unique_peaks.argtypes = [_ip, _dp, C.c_size_t, C.c_int, _ip, _dp]
        L.orc_find_peaks.restype = C.c_size_t
        L.orc_find_peaks.argtypes = [_dp, C.c_uint, C.c_double, C.c_int, C.c_float,
                                     C.c_float, C.c_float, C.c_int, _ip, _dp, _fp,
                                     C.c_size_t, C.POINTER(C.c_size_t)]
        L.orc_accel_list.restype = C.c_size_t
        L.orc_accel_list.argtypes = [C.c_float] * 4 + [C.c_size_t] + [C.c_float] * 5 + [
            _fp, C.c_size_t]
        for nm in ("orc_harmonic_distill", "orc_accel_distill", "orc_dm_distill"):
            getattr(L, nm).restype = C.c_size_t
        L.orc_harmonic_distill.argtypes = [C.c_void_p, C.c_size_t, C.c_float, C.c_float,
                                           C.c_int, _ip, _ip]
        L.orc_accel_distill.argtypes = [C.c_void_p, C.c_size_t, C.c_float, C.c_float,
                                        _ip, _ip]
        L.orc_dm_distill.argtypes = [C.c_void_p, C.c_size_t, C.c_float, _ip, _ip]
        L.orc_search_dm.restype = C.c_size_t
        L.orc_search_dm.argtypes = [_fp, C.c_size_t, C.POINTER(_Params), C.c_void_p,
                                    C.c_void_p, C.c_size_t, C.c_void_p]
        _lib = L
    return _lib


# ---------------------------------------------------------------- transforms
def rfft(x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.size
    out = np.zeros(2 * (n // 2 + 1), np.float64)
    if lib().orc_rfft(x, n, out):
        raise ValueError(f"unsupported transform length {n}")
    return out.view(np.complex128)


def irfft(X, n: int) -> np.ndarray:
    X = np.ascontiguousarray(np.asarray(X, dtype=np.complex128)).view(np.float64)
    out = np.zeros(n, np.float64)
    if lib().orc_irfft(np.ascontiguousarray(X), n, out):
        raise ValueError(f"unsupported transform length {n}")
    return out


# ---------------------------------------------------------------- resample
def accel_fact(acc: float, tsamp: float) -> float:
    return lib().orc_accel_fact(acc, tsamp)


def resampleII_index(n: int, acc: float, tsamp: float, fused: int = 1) -> np.ndarray:
    idx = np.zeros(n, np.uint64)
    lib().orc_resampleII_index(n, acc, tsamp, fused, idx)
    return idx


def resample_index(n: int, acc: float, tsamp: float, fused: int = 1) -> np.ndarray:
    idx = np.zeros(n, np.uint64)
    lib().orc_resample_index(n, acc, tsamp, fused, idx)
    return idx


def resampleII(x, acc: float, tsamp: float, fused: int = 1) -> np.ndarray:
    x = np.asarray(x, np.float64)
    return x[resampleII_index(x.size, acc, tsamp, fused).astype(np.int64)]


# ---------------------------------------------------------------- spectra
def _c2d(X):
    return np.ascontiguousarray(np.asarray(X, np.complex128)).view(np.float64)


def form_power(X) -> np.ndarray:
    Xd = _c2d(X)
    out = np.zeros(Xd.size // 2, np.float64)
    lib().orc_form_power(Xd, out.size, out)
    return out


def form_interbin(X) -> np.ndarray:
    Xd = _c2d(X)
    out = np.zeros(Xd.size // 2, np.float64)
    lib().orc_form_interbin(Xd, out.size, out)
    return out


def median_scrunch5(x) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros(max(1, x.size // 5), np.float64)
    n = lib().orc_median_scrunch5(x, x.size, out)
    return out[:n]


def linear_stretch(x, out_count: int) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros(out_count, np.float64)
    lib().orc_linear_stretch(x, x.size, out, out_count)
    return out


def stretch_overreads() -> int:
    return int(lib().orc_stretch_overreads())


def splice_points(nbins: int, bin_width: float, b5: float = 0.05, b25: float = 0.5):
    p5, p25 = C.c_int(), C.c_int()
    lib().orc_splice_points(nbins, bin_width, b5, b25, C.byref(p5), C.byref(p25))
    return p5.value, p25.value


def running_median(powers, bin_width: float, b5: float = 0.05, b25: float = 0.5):
    p = np.ascontiguousarray(powers, np.float64)
    out = np.zeros(p.size, np.float64)
    lib().orc_running_median(p, p.size, bin_width, b5, b25, out)
    return out


def deredden(X, median) -> np.ndarray:
    Xd = _c2d(X).copy()
    m = np.ascontiguousarray(median, np.float64)
    lib().orc_deredden(Xd, m, m.size)
    return Xd.view(np.complex128)


def zap_range(freq: float, width: float, bin_width: float, nbins: int):
    lo, hi = C.c_int(), C.c_int()
    lib().orc_zap_range(freq, width, bin_width, nbins, C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def zap(X, bin_width: float, freqs, widths) -> np.ndarray:
    Xd = _c2d(X).copy()
    f = np.ascontiguousarray(freqs, np.float32)
    w = np.ascontiguousarray(widths, np.float32)
    lib().orc_zap(Xd, Xd.size // 2, bin_width, f, w, f.size)
    return Xd.view(np.complex128)


def stats(x, first: int = 0):
    x = np.ascontiguousarray(x, np.float64)
    m, r, s = C.c_double(), C.c_double(), C.c_double()
    lib().orc_stats(x, x.size, first, C.byref(m), C.byref(r), C.byref(s))
    return m.value, r.value, s.value


def normalise(x, mean: float, sigma: float) -> np.ndarray:
    y = np.ascontiguousarray(x, np.float64).copy()
    lib().orc_normalise(y, y.size, mean, sigma)
    return y


def remove_baseline(x):
    y = np.ascontiguousarray(x, np.float64).copy()
    passes = lib().orc_remove_baseline(y, y.size)
    return y, passes


def harmonic_sums(p, nfolds: int) -> np.ndarray:
    p = np.ascontiguousarray(p, np.float64)
    out = np.zeros((nfolds, p.size), np.float64)
    if lib().orc_harmonic_sums(p, p.size, nfolds, out):
        raise ValueError("nfolds must be in 0..5")
    return out


def peak_range(nbins: int, bin_width: float, nh: int, min_freq: float, max_freq: float):
    s, e, f = C.c_int(), C.c_int(), C.c_float()
    lib().orc_peak_range(nbins, bin_width, nh, min_freq, max_freq, C.byref(s),
                         C.byref(e), C.byref(f))
    return s.value, e.value, f.value


def identify_unique_peaks(idx, snr, min_gap: int = 30):
    idx = np.ascontiguousarray(idx, np.int32)
    snr = np.ascontiguousarray(snr, np.float64)
    pi = np.zeros(max(1, idx.size), np.int32)
    ps = np.zeros(max(1, idx.size), np.float64)
    n = lib().orc_identify_unique_peaks(idx, snr, idx.size, min_gap, pi, ps)
    return pi[:n], ps[:n]


def find_peaks(spec, bin_width: float, nh: int, thresh: float, min_freq: float,
               max_freq: float, min_gap: int = 30):
    spec = np.ascontiguousarray(spec, np.float64)
    cap = max(1, spec.size)
    pi = np.zeros(cap, np.int32)
    ps = np.zeros(cap, np.float64)
    pf = np.zeros(cap, np.float32)
    nab = C.c_size_t()
    n = lib().orc_find_peaks(spec, spec.size, bin_width, nh, thresh, min_freq, max_freq,
                             min_gap, pi, ps, pf, cap, C.byref(nab))
    return pi[:n], ps[:n], pf[:n]


# ---------------------------------------------------------------- planning
def accel_list(acc_lo, acc_hi, tol, pulse_width_s, nsamps, tsamp, cfreq_hz, ch_bw_hz,
               dm, cdm) -> np.ndarray:
    args = (acc_lo, acc_hi, tol, pulse_width_s, nsamps, tsamp, cfreq_hz, ch_bw_hz, dm, cdm)
    n = lib().orc_accel_list(*args, np.zeros(1, np.float32), 0)
    out = np.zeros(n + 1, np.float32)
    n = lib().orc_accel_list(*args, out, out.size)
    return out[:n].copy()


def _cands_to_c(cands: np.ndarray):
    arr = np.ascontiguousarray(cands, dtype=CAND_DTYPE).copy()
    return arr, arr.ctypes.data


def harmonic_distill(cands, tol=1e-4, max_harm=16.0, fractional=True):
    arr, ptr = _cands_to_c(cands)
    keep = np.zeros(max(1, arr.size), np.int32)
    na = np.zeros(max(1, arr.size), np.int32)
    lib().orc_harmonic_distill(ptr, arr.size, tol, max_harm, int(fractional), keep, na)
    return arr[keep[:arr.size] == 1], arr, keep[:arr.size], na[:arr.size]


def accel_distill(cands, tobs, tol=1e-4):
    arr, ptr = _cands_to_c(cands)
    keep = np.zeros(max(1, arr.size), np.int32)
    na = np.zeros(max(1, arr.size), np.int32)
    lib().orc_accel_distill(ptr, arr.size, tobs, tol, keep, na)
    return arr[keep[:arr.size] == 1], arr, keep[:arr.size], na[:arr.size]


def dm_distill(cands, tol=1e-4):
    arr, ptr = _cands_to_c(cands)
    keep = np.zeros(max(1, arr.size), np.int32)
    na = np.zeros(max(1, arr.size), np.int32)
    lib().orc_dm_distill(ptr, arr.size, tol, keep, na)
    return arr[keep[:arr.size] == 1], arr, keep[:arr.size], na[:arr.size]


# ---------------------------------------------------------------- search
@dataclass
class SearchParams:
    """The parameters the reference's Worker reads (CmdLineOptions fields,
    include/utils/cmdline.hpp:6-41, with its defaults at :149-191)."""
    fft_size: int
    tsamp: float
    dm: float = 0.0
    cdm: float = 0.0
    dm_idx: int = 0
    acc_lo: float = 0.0
    acc_hi: float = 0.0
    acc_tol: float = 1.10
    acc_pulse_width: float = 64e-6
    cfreq: float = 1475.12e6
    ch_bw: float = 1.09e6
    nharmonics: int = 4
    min_snr: float = 9.0
    min_freq: float = 0.1
    max_freq: float = 1100.0
    min_gap: int = 30
    freq_tol: float = 1e-4
    max_harm: float = 16.0
    birdie_freqs: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    birdie_widths: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    resample_fused: int = 1


def search_dm(series, p: SearchParams, tap_trial: int = -1):
    """Per-trial harmonic-distilled candidates for one DM trial (all its
    acceleration trials, in trial order) and the acceleration-trial index of
    each.  With tap_trial >= 0 also returns that trial's intermediate
    buffers."""
    series = np.ascontiguousarray(series, np.float32)
    bf = np.ascontiguousarray(p.birdie_freqs, np.float32)
    bw = np.ascontiguousarray(p.birdie_widths, np.float32)
    cp = _Params(p.fft_size, p.tsamp, p.dm, p.cdm, p.dm_idx, p.acc_lo, p.acc_hi,
                 p.acc_tol, p.acc_pulse_width, p.cfreq, p.ch_bw, p.nharmonics,
                 p.min_snr, p.min_freq, p.max_freq, p.min_gap, p.freq_tol, p.max_harm,
                 bf.ctypes.data_as(C.POINTER(C.c_float)),
                 bw.ctypes.data_as(C.POINTER(C.c_float)), bf.size, p.resample_fused)
    N, B = p.fft_size, p.fft_size // 2 + 1
    taps = None
    bufs = {}
    if tap_trial >= 0:
        bufs = dict(tim_dered=np.zeros(N), tim_r=np.zeros(N), pspec=np.zeros(B),
                    sums=np.zeros(max(1, p.nharmonics) * B), median=np.zeros(B))
        dp = C.POINTER(C.c_double)
        taps = _Taps(tap_trial, *[bufs[k].ctypes.data_as(dp) for k in
                                  ("tim_dered", "tim_r", "pspec", "sums", "median")])
    cap = 1 << 16
    while True:
        out = np.zeros(cap, CAND_DTYPE)
        trial = np.zeros(cap, np.int32)
        n = lib().orc_search_dm(series, series.size, C.byref(cp), out.ctypes.data,
                                trial.ctypes.data, cap,
                                C.cast(C.pointer(taps), C.c_void_p) if taps else None)
        if n != (1 << 64) - 1:
            break
        if cap > (1 << 24):
            raise RuntimeError("oracle search failed")
        cap *= 4
    res = (out[:n].copy(), trial[:n].copy())
    if taps is not None:
        bufs["sums"] = bufs["sums"].reshape(max(1, p.nharmonics), B)[:p.nharmonics]
        bufs["stats"] = tuple(taps.stats)
        return res + (bufs,)
    return res


# ------------------------------------------------- FP32 CPU rendering
CPU_RENDER_PATH = os.path.join(HERE, "_build", "libcpu_render.so")
_cpu = None


def build_cpu_render() -> None:
    """Compile the FP32 CPU rendering (g++ against libtorch; about 30 s)."""
    subprocess.run(["make", "-s", "-C", HERE, "cpu"], check=True)


def cpu_render():
    global _cpu
    if _cpu is None:
        if not os.path.exists(CPU_RENDER_PATH):
            build_cpu_render()
        lib()  # the stage functions it links are the oracle's
        L = C.CDLL(CPU_RENDER_PATH)
        L.cpu_search_dm.restype = C.c_size_t
        L.cpu_search_dm.argtypes = [_fp, C.c_size_t, C.POINTER(_Params), C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_size_t, C.POINTER(C.c_double)]
        _cpu = L
    return _cpu


def cpu_search_dm(series, p: SearchParams, nthreads: int):
    """The FP32 CPU rendering of one DM trial on `nthreads` host threads:
    per-trial harmonic-distilled candidates (as search_dm), the trial index
    of each, and the wall time of the DM trial in seconds."""
    series = np.ascontiguousarray(series, np.float32)
    bf = np.ascontiguousarray(p.birdie_freqs, np.float32)
    bw = np.ascontiguousarray(p.birdie_widths, np.float32)
    cp = _Params(p.fft_size, p.tsamp, p.dm, p.cdm, p.dm_idx, p.acc_lo, p.acc_hi,
                 p.acc_tol, p.acc_pulse_width, p.cfreq, p.ch_bw, p.nharmonics,
                 p.min_snr, p.min_freq, p.max_freq, p.min_gap, p.freq_tol, p.max_harm,
                 bf.ctypes.data_as(C.POINTER(C.c_float)),
                 bw.ctypes.data_as(C.POINTER(C.c_float)), bf.size, p.resample_fused)
    cap = 1 << 16
    sec = C.c_double()
    while True:
        out = np.zeros(cap, CAND_DTYPE)
        trial = np.zeros(cap, np.int32)
        n = cpu_render().cpu_search_dm(series, series.size, C.byref(cp), int(nthreads),
                                       out.ctypes.data, trial.ctypes.data, cap, C.byref(sec))
        if n != (1 << 64) - 1:
            break
        if cap > (1 << 24):
            raise RuntimeError("CPU rendering failed")
        cap *= 4
    return out[:n].copy(), trial[:n].copy(), sec.value


# ---------------------------------------------------------------- reference
_ref_host = None
_ref_gpu = None


def ref_host():
    """The reference's own host classes (AccelerationPlan, distillers)."""
    global _ref_host
    if _ref_host is None:
        if not os.path.exists(REF_HOST_PATH):
            raise FileNotFoundError(REF_HOST_PATH)
        L = C.CDLL(REF_HOST_PATH)
        L.ref_accel_list.restype = C.c_size_t
        L.ref_accel_list.argtypes = [C.c_float] * 4 + [C.c_size_t] + [C.c_float] * 5 + [
            _fp, C.c_size_t]
        L.ref_distill.restype = C.c_size_t
        L.ref_distill.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.c_float, C.c_float,
                                  C.c_float, C.c_int, C.c_int, C.c_void_p, _ip]
        vp, sz, f = C.c_void_p, C.c_size_t, C.c_float
        L.ref_distill_forest.restype = sz
        L.ref_distill_forest.argtypes = [C.c_int, vp, vp, sz, f, f, f, C.c_int, C.c_int, vp, vp,
                                         sz]
        L.ref_score_forest.restype = sz
        L.ref_score_forest.argtypes = [vp, vp, sz, f, f, f, f, vp]
        L.ref_write_binary.restype = sz
        L.ref_write_binary.argtypes = [C.c_char_p, C.c_char_p, vp, vp, sz, vp]
        L.ref_overview_text.restype = sz
        L.ref_overview_text.argtypes = [vp, sz, vp, sz, f, vp, vp, sz, vp, f, f, f, f, vp, sz]
        _ref_host = L
    return _ref_host


def ref_accel_list(*args) -> np.ndarray:
    L = ref_host()
    n = L.ref_accel_list(*args, np.zeros(1, np.float32), 0)
    out = np.zeros(max(1, n), np.float32)
    L.ref_accel_list(*args, out, out.size)
    return out[:n]


def ref_distill(kind: int, cands, tol=1e-4, max_harm=16.0, tobs=0.0, keep_related=False,
                fractional=True):
    arr = np.ascontiguousarray(cands, dtype=CAND_DTYPE).copy()
    out = np.zeros(max(1, arr.size), CAND_DTYPE)
    na = np.zeros(max(1, arr.size), np.int32)
    n = ref_host().ref_distill(kind, arr.ctypes.data, arr.size, tol, max_harm, tobs,
                               int(keep_related), int(fractional), out.ctypes.data, na)
    return out[:n], na[:n]


SCORE_DTYPE = np.dtype([("is_physical", "<i4"), ("is_adjacent", "<i4"),
                        ("ddm_count_ratio", "<f4"), ("ddm_snr_ratio", "<f4"),
                        ("nassoc", "<i4")])


def ref_distill_forest(kind, nodes, sizes, tol=1e-4, max_harm=16.0, tobs=0.0,
                       keep_related=True, fractional=False):
    """The reference's distillers on candidate trees (a forest: nodes in
    depth-first order with subtree sizes); returns the survivors' forest."""
    a = np.ascontiguousarray(nodes, CAND_DTYPE)
    sz = np.ascontiguousarray(sizes, np.int32)
    L = ref_host()
    args = (kind, a.ctypes.data, sz.ctypes.data, a.size, tol, max_harm, tobs,
            int(keep_related), int(fractional))
    n = L.ref_distill_forest(*args, None, None, 0)
    out = np.zeros(max(1, n), CAND_DTYPE)
    osz = np.zeros(max(1, n), np.int32)
    L.ref_distill_forest(*args, out.ctypes.data, osz.ctypes.data, out.size)
    return out[:n], osz[:n]


def _nroots(sizes):
    i, k = 0, 0
    while i < len(sizes):
        i += int(sizes[i])
        k += 1
    return k


def ref_score_forest(nodes, sizes, tsamp, cfreq, foff, bw):
    a = np.ascontiguousarray(nodes, CAND_DTYPE)
    sz = np.ascontiguousarray(sizes, np.int32)
    out = np.zeros(max(1, _nroots(sz)), SCORE_DTYPE)
    n = ref_host().ref_score_forest(a.ctypes.data, sz.ctypes.data, a.size, tsamp, cfreq, foff, bw,
                                    out.ctypes.data)
    return out[:n]


def ref_write_binary(directory, filename, nodes, sizes):
    a = np.ascontiguousarray(nodes, CAND_DTYPE)
    sz = np.ascontiguousarray(sizes, np.int32)
    off = np.zeros(max(1, _nroots(sz)), np.int64)
    n = ref_host().ref_write_binary(directory.encode(), filename.encode(), a.ctypes.data,
                                    sz.ctypes.data, a.size, off.ctypes.data)
    return off[:n]


def ref_overview_text(dms, accs, cdm, nodes, sizes, offsets, tsamp, cfreq, foff, bw) -> str:
    d = np.ascontiguousarray(dms, np.float32)
    ac = np.ascontiguousarray(accs, np.float32)
    a = np.ascontiguousarray(nodes, CAND_DTYPE)
    sz = np.ascontiguousarray(sizes, np.int32)
    off = np.ascontiguousarray(offsets, np.int64)
    L = ref_host()
    args = (d.ctypes.data, d.size, ac.ctypes.data, ac.size, cdm, a.ctypes.data, sz.ctypes.data,
            a.size, off.ctypes.data, tsamp, cfreq, foff, bw)
    n = L.ref_overview_text(*args, None, 0)
    buf = C.create_string_buffer(n + 1)
    L.ref_overview_text(*args, buf, n + 1)
    return buf.value.decode("latin-1")


class _RefArgs(C.Structure):
    _fields_ = [("cdm", C.c_float), ("acc_start", C.c_float), ("acc_end", C.c_float),
                ("acc_tol", C.c_float), ("acc_pulse_width_us", C.c_float),
                ("cfreq_hz", C.c_float), ("ch_bw_hz", C.c_float),
                ("nharmonics", C.c_int), ("min_snr", C.c_float), ("min_freq", C.c_float),
                ("max_freq", C.c_float), ("max_harm", C.c_int), ("freq_tol", C.c_float),
                ("zapfile", C.c_char_p)]


def ref_gpu():
    """The reference's own CUDA implementation (needs a GPU)."""
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(REF_GPU_PATH):
            raise FileNotFoundError(REF_GPU_PATH)
        L = C.CDLL(REF_GPU_PATH)
        for nm in ("ref_resampleII", "ref_resample"):
            getattr(L, nm).argtypes = [_fp, _fp, C.c_size_t, C.c_float, C.c_float]
        L.ref_fft_r2c.argtypes = [_fp, C.c_size_t, _fp]
        L.ref_fft_c2r.argtypes = [_fp, C.c_size_t, _fp]
        L.ref_form.argtypes = [_fp, C.c_size_t, C.c_int, _fp]
        L.ref_running_median.argtypes = [_fp, C.c_size_t, C.c_double, _fp]
        L.ref_deredden.argtypes = [_fp, _fp, C.c_size_t, C.c_double]
        L.ref_zap.argtypes = [_fp, C.c_size_t, C.c_double, C.c_char_p]
        L.ref_stats.argtypes = [_fp, C.c_size_t, C.POINTER(C.c_float),
                                C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.ref_normalise.argtypes = [_fp, C.c_size_t, C.c_float, C.c_float]
        L.ref_remove_baseline.argtypes = [_fp, C.c_size_t]
        L.ref_harmonic_sums.argtypes = [_fp, C.c_size_t, C.c_int, _fp]
        L.ref_find_candidates.argtypes = [_fp, C.c_size_t, C.c_double, C.c_int, C.c_float,
                                          C.c_float, C.c_float, C.c_int, _fp, _fp,
                                          C.c_size_t, C.POINTER(C.c_size_t)]
        L.ref_worker_search.argtypes = [_fp, C.c_size_t, C.c_size_t, C.c_float, _fp,
                                        C.c_size_t, C.POINTER(_RefArgs), C.c_void_p, _ip,
                                        C.c_size_t, C.POINTER(C.c_size_t)]
        _ref_gpu = L
    return _ref_gpu


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what} failed with status {rc}")


def ref_resampleII(x, acc, tsamp):
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    _chk(ref_gpu().ref_resampleII(x, out, x.size, acc, tsamp), "resampleII")
    return out


def ref_copy_from_host_8bit(x) -> np.ndarray:
    """The reference's ReusableDeviceTimeSeries<float, unsigned char | char>
    ::copy_from_host of a uint8 or int8 host array (its conversion_kernel)."""
    x = np.ascontiguousarray(x)
    if x.dtype not in (np.uint8, np.int8):
        raise TypeError("uint8 or int8 samples")
    out = np.zeros(x.size, np.float32)
    L = ref_gpu()
    fn = L.ref_copy_from_host_u8 if x.dtype == np.uint8 else L.ref_copy_from_host_i8
    fn.restype = C.c_int
    _chk(fn(x.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p), C.c_size_t(x.size)),
         "copy_from_host")
    return out


def ref_resample(x, acc, tsamp):
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    _chk(ref_gpu().ref_resample(x, out, x.size, acc, tsamp), "resample")
    return out


def ref_fft_r2c(x):
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros(2 * (x.size // 2 + 1), np.float32)
    _chk(ref_gpu().ref_fft_r2c(x, x.size, out), "fft_r2c")
    return out.view(np.complex64)


def ref_fft_c2r(X, n):
    X = np.ascontiguousarray(np.asarray(X, np.complex64)).view(np.float32)
    out = np.zeros(n, np.float32)
    _chk(ref_gpu().ref_fft_c2r(np.ascontiguousarray(X), n, out), "fft_c2r")
    return out


def ref_form(X, interbin: bool):
    Xf = np.ascontiguousarray(np.asarray(X, np.complex64)).view(np.float32)
    out = np.zeros(Xf.size // 2, np.float32)
    _chk(ref_gpu().ref_form(np.ascontiguousarray(Xf), out.size, int(interbin), out), "form")
    return out


def ref_running_median(powers, bin_width):
    p = np.ascontiguousarray(powers, np.float32)
    out = np.zeros_like(p)
    _chk(ref_gpu().ref_running_median(p, p.size, bin_width, out), "running_median")
    return out


def ref_deredden(X, powers, bin_width):
    Xf = np.ascontiguousarray(np.asarray(X, np.complex64)).view(np.float32).copy()
    p = np.ascontiguousarray(powers, np.float32)
    _chk(ref_gpu().ref_deredden(Xf, p, p.size, bin_width), "deredden")
    return Xf.view(np.complex64)


def ref_zap(X, bin_width, zapfile: str):
    Xf = np.ascontiguousarray(np.asarray(X, np.complex64)).view(np.float32).copy()
    _chk(ref_gpu().ref_zap(Xf, Xf.size // 2, bin_width, zapfile.encode()), "zap")
    return Xf.view(np.complex64)


def ref_stats(x):
    x = np.ascontiguousarray(x, np.float32)
    m, r, s = C.c_float(), C.c_float(), C.c_float()
    _chk(ref_gpu().ref_stats(x, x.size, C.byref(m), C.byref(r), C.byref(s)), "stats")
    return m.value, r.value, s.value


def ref_normalise(x, mean, sd):
    y = np.ascontiguousarray(x, np.float32).copy()
    _chk(ref_gpu().ref_normalise(y, y.size, mean, sd), "normalise")
    return y


def ref_remove_baseline(x):
    y = np.ascontiguousarray(x, np.float32).copy()
    _chk(ref_gpu().ref_remove_baseline(y, y.size), "remove_baseline")
    return y


def ref_harmonic_sums(p, nfolds):
    p = np.ascontiguousarray(p, np.float32)
    out = np.zeros((nfolds, p.size), np.float32)
    _chk(ref_gpu().ref_harmonic_sums(p, p.size, nfolds, out), "harmonic_sums")
    return out


def ref_find_candidates(spec, bin_width, nh, thresh, min_freq, max_freq, min_gap=30):
    spec = np.ascontiguousarray(spec, np.float32)
    cap = 1 << 20
    snr = np.zeros(cap, np.float32)
    freq = np.zeros(cap, np.float32)
    n = C.c_size_t()
    _chk(ref_gpu().ref_find_candidates(spec, spec.size, bin_width, nh, thresh, min_freq,
                                       max_freq, min_gap, snr, freq, cap, C.byref(n)),
         "find_candidates")
    return snr[:n.value].copy(), freq[:n.value].copy()


def ref_worker_search_forest(series2d, tsamp, dms, fft_size, p: SearchParams,
                             zapfile: str = ""):
    """The same run as ref_worker_search; the per-DM candidates with their
    association trees, as a forest (nodes, subtree sizes)."""
    s = np.ascontiguousarray(series2d, np.float32)
    ndm, nsamps = s.shape
    a = _RefArgs(p.cdm, p.acc_lo, p.acc_hi, p.acc_tol, p.acc_pulse_width * 1e6, p.cfreq,
                 p.ch_bw, p.nharmonics, p.min_snr, p.min_freq, p.max_freq,
                 int(p.max_harm), p.freq_tol, zapfile.encode())
    cap = 1 << 20
    out = np.zeros(cap, CAND_DTYPE)
    sz = np.zeros(cap, np.int32)
    n = C.c_size_t()
    L = ref_gpu()
    L.ref_worker_search_forest.restype = C.c_int
    _chk(L.ref_worker_search_forest(s.reshape(-1).ctypes.data_as(C.c_void_p), C.c_size_t(ndm),
                                    C.c_size_t(nsamps), C.c_float(tsamp),
                                    np.ascontiguousarray(dms, np.float32).ctypes.data_as(
                                        C.c_void_p), C.c_size_t(fft_size), C.byref(a),
                                    out.ctypes.data_as(C.c_void_p), sz.ctypes.data_as(C.c_void_p),
                                    C.c_size_t(cap), C.byref(n)),
         "worker_search_forest")
    return out[:n.value].copy(), sz[:n.value].copy()


def ref_worker_search(series2d, tsamp, dms, fft_size, p: SearchParams, zapfile: str = ""):
    """The reference's unmodified Worker::start over a block of DM trials;
    returns its per-DM acceleration-distilled candidates and their
    association counts."""
    s = np.ascontiguousarray(series2d, np.float32)
    ndm, nsamps = s.shape
    a = _RefArgs(p.cdm, p.acc_lo, p.acc_hi, p.acc_tol, p.acc_pulse_width * 1e6, p.cfreq,
                 p.ch_bw, p.nharmonics, p.min_snr, p.min_freq, p.max_freq,
                 int(p.max_harm), p.freq_tol, zapfile.encode())
    cap = 1 << 20
    out = np.zeros(cap, CAND_DTYPE)
    na = np.zeros(cap, np.int32)
    n = C.c_size_t()
    _chk(ref_gpu().ref_worker_search(s.reshape(-1), ndm, nsamps, tsamp,
                                     np.ascontiguousarray(dms, np.float32), fft_size,
                                     C.byref(a), out.ctypes.data, na, cap, C.byref(n)),
         "worker_search")
    return out[:n.value].copy(), na[:n.value].copy()


# ---------------------------------------------------------------- dedispersion
def _dedisp_lib():
    L = lib()
    if not getattr(L, "_dedisp_ready", False):
        L.orc_delay_table.argtypes = [C.c_size_t, C.c_float, C.c_float, C.c_float, _fp]
        L.orc_dm_list.restype = C.c_size_t
        L.orc_dm_list.argtypes = [C.c_size_t] + [C.c_float] * 7 + [_fp, C.c_size_t]
        L.orc_max_delay.restype = C.c_size_t
        L.orc_max_delay.argtypes = [_fp, C.c_size_t, _fp, C.c_size_t]
        L.orc_dedisperse.restype = C.c_int
        L.orc_dedisperse.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_int, _fp, _fp,
                                     C.c_size_t, C.c_void_p, C.c_int, _fp, C.c_size_t]
        L.orc_sigproc_value.restype = C.c_uint
        L.orc_sigproc_value.argtypes = [C.c_void_p, C.c_size_t, C.c_int]
        L._dedisp_ready = True
    return L


def delay_table(nchans, tsamp, fch1, foff) -> np.ndarray:
    out = np.zeros(nchans, np.float32)
    _dedisp_lib().orc_delay_table(nchans, tsamp, fch1, foff, out)
    return out


def dm_list(nchans, tsamp, fch1, foff, dm_start, dm_end, width_us, tol) -> np.ndarray:
    L = _dedisp_lib()
    args = (nchans, tsamp, fch1, foff, dm_start, dm_end, width_us, tol)
    n = L.orc_dm_list(*args, np.zeros(1, np.float32), 0)
    out = np.zeros(n, np.float32)
    L.orc_dm_list(*args, out, n)
    return out


def max_delay(delays, dms) -> int:
    d = np.ascontiguousarray(delays, np.float32)
    m = np.ascontiguousarray(dms, np.float32)
    return int(_dedisp_lib().orc_max_delay(d, d.size, m, m.size))


def dedisperse(rows, nbits: int, nchans: int, delays, dms, killmask=None, raw=False):
    """rows: (nsamps, nchans*nbits/8) packed uint8 SIGPROC rows.  Returns
    (ndm, nsamps - max_delay) float32."""
    rows = np.ascontiguousarray(rows, np.uint8)
    d = np.ascontiguousarray(delays, np.float32)
    m = np.ascontiguousarray(dms, np.float32)
    ns = rows.shape[0]
    md = max_delay(d, m)
    out = np.zeros((m.size, ns - md), np.float32)
    km = None if killmask is None else np.ascontiguousarray(killmask, np.int32)
    rc = _dedisp_lib().orc_dedisperse(rows.ctypes.data, ns, nchans, nbits, d, m, m.size,
                                      None if km is None else km.ctypes.data, int(raw), out,
                                      out.shape[1])
    if rc:
        raise ValueError("orc_dedisperse: the samples do not exceed the maximum delay")
    return out


def unpack_rows(rows, nchans: int, nbits: int) -> np.ndarray:
    """Packed SIGPROC rows -> (nsamps, nchans) unsigned samples (numpy
    restatement of orc_sigproc_value for whole arrays)."""
    rows = np.ascontiguousarray(rows, np.uint8)
    if nbits == 8:
        return rows[:, :nchans].astype(np.uint32)
    if nbits == 16:
        return rows.view("<u2")[:, :nchans].astype(np.uint32)
    per = 8 // nbits
    mask = (1 << nbits) - 1
    out = np.zeros((rows.shape[0], nchans), np.uint32)
    for k in range(per):
        out[:, k::per] = (rows[:, :nchans // per] >> (k * nbits)) & mask
    return out


def parse_sigproc_header(path: str) -> dict:
    """Independent SIGPROC header parse (keyword, typed value) in Python,
    restating read_header (include/data_types/header.hpp:339-403)."""
    import struct
    ints = {"nchans", "telescope_id", "machine_id", "data_type", "ibeam", "nbeams", "nbits",
            "barycentric", "pulsarcentric", "nbins", "nsamples", "nifs", "npuls"}
    dbls = {"az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "period", "fch1",
            "foff", "refdm"}
    data = open(path, "rb").read()
    pos = 0

    def rs():
        nonlocal pos
        n = struct.unpack_from("<i", data, pos)[0]
        pos += 4
        s = data[pos:pos + n].decode()
        pos += n
        return s

    assert rs() == "HEADER_START"
    out = {}
    while True:
        k = rs()
        if k == "HEADER_END":
            break
        if k in ("source_name", "rawdatafile"):
            out[k] = rs()
        elif k in ints:
            out[k] = struct.unpack_from("<i", data, pos)[0]
            pos += 4
        elif k in dbls:
            out[k] = struct.unpack_from("<d", data, pos)[0]
            pos += 8
        elif k == "signed":
            out["signed_data"] = data[pos]
            pos += 1
    out["header_size"] = pos
    if not out.get("nsamples"):
        out["nsamples"] = (len(data) - pos) // out["nchans"] * 8 // out["nbits"]
    return out


_REF_HDR_KEYS = ["az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "period",
                 "fch1", "foff", "refdm", "nchans", "telescope_id", "machine_id", "data_type",
                 "ibeam", "nbeams", "nbits", "barycentric", "pulsarcentric", "nbins",
                 "nsamples", "nifs", "npuls", "signed_data", "header_size"]


def ref_sigproc_header(path: str) -> dict:
    """The reference's own read_header on `path` (oracle/_ref)."""
    L = ref_host()
    fn = L.ref_sigproc_header
    fn.restype = C.c_int
    fn.argtypes = [C.c_char_p, _dp, C.c_char_p, C.c_char_p]
    v = np.zeros(25, np.float64)
    sn = C.create_string_buffer(80)
    rd = C.create_string_buffer(80)
    if fn(path.encode(), v, sn, rd):
        raise OSError(path)
    out = dict(zip(_REF_HDR_KEYS, v.tolist()))
    out["source_name"] = sn.value.decode()
    out["rawdatafile"] = rd.value.decode()
    return out


def ref_filterbank_gulp(path: str, seg_start: int, seg_n: int, start: int, n: int,
                        row_bytes: int):
    """SigprocFilterbank(path, seg_start, seg_n).load_gulp(start, n): the
    bytes read and [tsamp, fch1, foff, cfreq, start, end, effective, total,
    pepoch at size 2^16]."""
    L = ref_host()
    fn = L.ref_filterbank_gulp
    fn.restype = C.c_size_t
    fn.argtypes = [C.c_char_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p,
                   C.c_size_t, _dp]
    out = np.zeros(max(1, n * row_bytes), np.uint8)
    meta = np.zeros(9, np.float64)
    got = fn(path.encode(), seg_start, seg_n, start, n, out.ctypes.data, out.size, meta)
    return out[:got * row_bytes], meta


def ref_write_timeseries(outdir: str, stem: str, block, dms, idx: int, hd, hi,
                         source_name: str) -> int:
    """The reference's DispersionTrials::write_timeseries_to_file (host code
    of oracle/_ref/libpeasoup_ref_gpu.so; no device call)."""
    if not os.path.exists(REF_GPU_PATH):
        raise FileNotFoundError(REF_GPU_PATH)
    L = C.CDLL(REF_GPU_PATH)
    f = L.ref_write_timeseries
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                  C.c_size_t, C.c_void_p, C.c_void_p, C.c_char_p]
    b = np.ascontiguousarray(block, np.float32)
    d = np.ascontiguousarray(dms, np.float32)
    hd = np.ascontiguousarray(hd, np.float64)
    hi = np.ascontiguousarray(hi, np.int32)
    return f(outdir.encode(), stem.encode(), b.ctypes.data, b.shape[1], d.ctypes.data, d.size,
             idx, hd.ctypes.data, hi.ctypes.data, source_name.encode())
