"""Python mirror of Peasoup's transform/operator API for the acceleration
search path, backed by the B200 kernels of libpeasoup_b200.so.

Class and method names, argument meaning and error behaviour follow the
reference's C++ headers (include/transforms/*.hpp, include/utils/stats.hpp,
include/data_types/{timeseries,fourierseries,candidates}.hpp,
include/utils/utils.hpp).  Device buffers are torch CUDA tensors (device
memory and stream plumbing only); every computation is a call into the
library.  Failures raise PsxError (a RuntimeError), as the reference
raises std::runtime_error.  Calls are asynchronous on torch's current CUDA
stream except where a host value is returned.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import Candidate as _CandPOD
from ._lib import PsxError, check, load

__all__ = [
    "PsxError", "DeviceTimeSeries", "DeviceFourierSeries", "DevicePowerSpectrum",
    "HarmonicSums", "TimeDomainResampler", "CuFFTerC2C", "CuFFTerR2C", "CuFFTerC2R",
    "SpectrumFormer",
    "Dereddener", "Zapper", "stats", "normalise", "SpectrumNormaliser", "HarmonicFolder",
    "PeakFinder", "Candidate", "CandidateCollection", "SpectrumCandidates",
    "HarmonicDistiller", "AccelerationDistiller", "DMDistiller", "AccelerationPlan",
]


def _stream() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor) -> C.c_void_p:
    if not t.is_cuda:
        raise PsxError(_lib.PSX_ERR_INVALID, "buffer", "expected a CUDA tensor")
    return C.c_void_p(t.data_ptr())


def _require_cuda():
    if not torch.cuda.is_available():
        raise PsxError(_lib.PSX_ERR_CUDA, "device", "no CUDA device (no CPU fallback)")


# --------------------------------------------------------------- containers
class DeviceTimeSeries:
    """include/data_types/timeseries.hpp:237-315: float samples on the GPU."""

    def __init__(self, nsamps: int, tsamp: float = 0.0, data: Optional[torch.Tensor] = None):
        _require_cuda()
        self.nsamps = int(nsamps)
        self.tsamp = float(tsamp)
        self.data = data if data is not None else torch.zeros(
            self.nsamps, dtype=torch.float32, device="cuda")

    @classmethod
    def from_host(cls, samples, tsamp: float) -> "DeviceTimeSeries":
        a = np.ascontiguousarray(samples, dtype=np.float32)
        return cls(a.size, tsamp, torch.from_numpy(a).cuda())

    def get_data(self) -> torch.Tensor:
        return self.data

    def get_nsamps(self) -> int:
        return self.nsamps

    def get_tsamp(self) -> float:
        return self.tsamp

    def set_tsamp(self, tsamp: float) -> None:
        self.tsamp = float(tsamp)

    def remove_baseline(self, nsamps: int = 0) -> int:
        """timeseries.hpp:282-287; returns the number of mean-removal passes."""
        n = nsamps or self.nsamps
        passes = C.c_int()
        check(load().psx_remove_baseline(_ptr(self.data), n, C.byref(passes), _stream()),
              "remove_baseline")
        return passes.value

    def fill(self, start: int, end: int, value: float) -> None:
        """timeseries.hpp:296-304."""
        if end > self.nsamps:
            raise PsxError(_lib.PSX_ERR_INVALID, "DeviceTimeSeries::fill",
                           "bad end value requested")
        if end > start:
            check(load().psx_fill(C.c_void_p(self.data.data_ptr() + 4 * start), end - start,
                                  value, _stream()), "fill")


class _FrequencySeries:
    def __init__(self, nbins: int, bin_width: float):
        self.nbins = int(nbins)
        self.bin_width = float(bin_width)

    def get_nbins(self) -> int:
        return self.nbins

    def get_bin_width(self) -> float:
        return self.bin_width

    def set_bin_width(self, bw: float) -> None:
        self.bin_width = float(bw)


class DeviceFourierSeries(_FrequencySeries):
    """fourierseries.hpp:136-141: complex spectrum (interleaved float pairs)."""

    def __init__(self, nbins: int, bin_width: float, data: Optional[torch.Tensor] = None):
        _require_cuda()
        super().__init__(nbins, bin_width)
        self.data = data if data is not None else torch.zeros(
            2 * self.nbins, dtype=torch.float32, device="cuda")

    def get_data(self) -> torch.Tensor:
        return self.data

    def complex(self) -> torch.Tensor:
        return torch.view_as_complex(self.data.view(-1, 2))


class DevicePowerSpectrum(_FrequencySeries):
    """fourierseries.hpp:143-160: real spectrum with harmonic number nh."""

    def __init__(self, nbins, bin_width: float = 0.0, nh: int = 0,
                 data: Optional[torch.Tensor] = None):
        _require_cuda()
        if isinstance(nbins, _FrequencySeries):  # DevicePowerSpectrum(other, nh)
            other = nbins
            super().__init__(other.get_nbins(), other.get_bin_width())
            nh = int(bin_width) if bin_width else nh
        else:
            super().__init__(nbins, bin_width)
        self.nh = int(nh)
        self.data = data if data is not None else torch.zeros(
            self.nbins, dtype=torch.float32, device="cuda")

    def get_data(self) -> torch.Tensor:
        return self.data

    def get_nh(self) -> int:
        return self.nh

    def set_nh(self, nh: int) -> None:
        self.nh = int(nh)


class HarmonicSums:
    """fourierseries.hpp:162-188: nfolds spectra, fold h has nh = h+1."""

    def __init__(self, fold0: DevicePowerSpectrum, nfolds: int):
        self.folds = [DevicePowerSpectrum(fold0, ii + 1) for ii in range(int(nfolds))]

    def size(self) -> int:
        return len(self.folds)

    def __len__(self) -> int:
        return len(self.folds)

    def __getitem__(self, ii: int) -> DevicePowerSpectrum:
        return self.folds[ii]


# --------------------------------------------------------------- transforms
class TimeDomainResampler:
    """include/transforms/resampler.hpp:7-34."""

    def resample(self, input: DeviceTimeSeries, output: DeviceTimeSeries, size: int,
                 acc: float) -> None:
        check(load().psx_resample(_ptr(input.data), _ptr(output.data), int(size), acc,
                                  input.get_tsamp(), _stream()), "resample")

    def resampleII(self, input: DeviceTimeSeries, output: DeviceTimeSeries, size: int,
                   acc: float) -> None:
        check(load().psx_resampleII(_ptr(input.data), _ptr(output.data), int(size), acc,
                                    input.get_tsamp(), _stream()), "resampleII")


class _CuFFTer:
    kind = _lib.PSX_FFT_R2C

    def __init__(self, size: int, batch: int = 1):
        _require_cuda()
        self.size = int(size)
        self._plan = C.c_void_p()
        check(load().psx_fft_plan_create(C.byref(self._plan), self.size, int(batch), self.kind),
              type(self).__name__)

    def get_resolution(self, tsamp: float) -> float:
        return 1.0 / (self.size * tsamp)

    def get_output_size(self) -> int:
        return self.size // 2 + 1

    def _exec(self, a: torch.Tensor, b: torch.Tensor, where: str) -> None:
        check(load().psx_fft_exec(self._plan, _ptr(a), _ptr(b), _stream()), where)

    def __del__(self):
        try:
            if self._plan:
                torch.cuda.synchronize()
                load().psx_fft_plan_destroy(self._plan)
                self._plan = C.c_void_p()
        except Exception:
            pass


class CuFFTerC2C(_CuFFTer):
    """include/transforms/ffter.hpp:33-53: unnormalised complex transform;
    direction -1 (CUFFT_FORWARD) or +1 (CUFFT_INVERSE) per call."""
    kind = _lib.PSX_FFT_C2C

    def get_output_size(self) -> int:
        return self.size

    def execute(self, input, output, direction: int) -> None:
        a = input.get_data() if hasattr(input, "get_data") else input
        b = output.get_data() if hasattr(output, "get_data") else output
        check(load().psx_fft_exec_c2c(self._plan, _ptr(a), _ptr(b), int(direction), _stream()),
              "CuFFTerC2C::execute")


class CuFFTerR2C(_CuFFTer):
    """include/transforms/ffter.hpp:54-80: unnormalised R2C."""
    kind = _lib.PSX_FFT_R2C

    def execute(self, tim, fseries) -> None:
        a = tim.get_data() if hasattr(tim, "get_data") else tim
        b = fseries.get_data() if hasattr(fseries, "get_data") else fseries
        self._exec(a, b, "CuFFTerR2C::execute")


class CuFFTerC2R(_CuFFTer):
    """include/transforms/ffter.hpp:82-110: unnormalised C2R."""
    kind = _lib.PSX_FFT_C2R

    def get_output_size(self) -> int:
        return self.size

    def execute(self, fseries, tim) -> None:
        a = fseries.get_data() if hasattr(fseries, "get_data") else fseries
        b = tim.get_data() if hasattr(tim, "get_data") else tim
        self._exec(a, b, "CuFFTerC2R::execute")


class SpectrumFormer:
    """include/transforms/spectrumformer.hpp:6-24."""

    def form_interpolated(self, input: DeviceFourierSeries, output: DevicePowerSpectrum) -> None:
        check(load().psx_form_power_series(_ptr(input.data), _ptr(output.data),
                                           input.get_nbins(), 1, _stream()), "form_interpolated")

    def form(self, input: DeviceFourierSeries, output: DevicePowerSpectrum) -> None:
        check(load().psx_form_power_series(_ptr(input.data), _ptr(output.data),
                                           input.get_nbins(), 0, _stream()), "form")


class Dereddener:
    """include/transforms/dereddener.hpp:10-68: 5/25/125-bin running median."""

    def __init__(self, size: int):
        _require_cuda()
        self.size = int(size)
        self.median = torch.zeros(self.size, dtype=torch.float32, device="cuda")
        nbytes = load().psx_running_median_scratch_bytes(self.size)
        self._scratch = torch.zeros((nbytes + 3) // 4, dtype=torch.float32, device="cuda")

    def calculate_median(self, powers: DevicePowerSpectrum, boundary_5_freq: float = 0.05,
                         boundary_25_freq: float = 0.5) -> None:
        if powers.get_nbins() != self.size:
            raise PsxError(_lib.PSX_ERR_INVALID, "Dereddener",
                           "Bad data length given to running_median()")
        check(load().psx_running_median(_ptr(powers.data), self.size, powers.get_bin_width(),
                                        boundary_5_freq, boundary_25_freq, _ptr(self.median),
                                        _ptr(self._scratch), _stream()), "calculate_median")

    def deredden(self, spectrum: DeviceFourierSeries) -> None:
        check(load().psx_divide_c_by_f(_ptr(spectrum.data), _ptr(self.median),
                                       spectrum.get_nbins(), _stream()), "deredden")


class Zapper:
    """include/transforms/birdiezapper.hpp:11-73: zap list of "freq width"."""

    def __init__(self, zaplist: str):
        _require_cuda()
        self.birdies = np.zeros(0, np.float32)
        self.widths = np.zeros(0, np.float32)
        self.append_from_file(zaplist)

    @classmethod
    def from_arrays(cls, freqs, widths) -> "Zapper":
        z = cls.__new__(cls)
        z.birdies = np.ascontiguousarray(freqs, np.float32)
        z.widths = np.ascontiguousarray(widths, np.float32)
        z._upload()
        return z

    def append_from_file(self, zaplist: str) -> None:
        L = load()
        n = C.c_size_t()
        check(L.psx_read_zaplist(zaplist.encode(), None, None, 0, C.byref(n)), "Zapper")
        f = np.zeros(max(1, n.value), np.float32)
        w = np.zeros(max(1, n.value), np.float32)
        check(L.psx_read_zaplist(zaplist.encode(), f.ctypes.data, w.ctypes.data, f.size,
                                 C.byref(n)), "Zapper")
        self.birdies = np.concatenate([self.birdies, f[:n.value]])
        self.widths = np.concatenate([self.widths, w[:n.value]])
        self._upload()

    def _upload(self) -> None:
        self.d_birdies = torch.from_numpy(self.birdies.copy()).cuda()
        self.d_widths = torch.from_numpy(self.widths.copy()).cuda()

    def zap(self, fseries: DeviceFourierSeries) -> None:
        self.zap_raw(fseries.data, np.float32(fseries.get_bin_width()), fseries.get_nbins())

    def zap_raw(self, data: torch.Tensor, bin_width: float, nbins: int) -> None:
        if self.birdies.size == 0:
            return
        check(load().psx_zap_birdies(_ptr(data), _ptr(self.d_birdies), _ptr(self.d_widths),
                                     float(np.float32(bin_width)), self.birdies.size, nbins,
                                     _stream()), "zap")


class stats:  # noqa: N801  (namespace in the reference: include/utils/stats.hpp)
    """include/utils/stats.hpp:6-43."""

    @staticmethod
    def stats(data: torch.Tensor, nsamps: int, first_samp: int = 0):
        """Returns (mean, rms, std) of data[first_samp:nsamps]."""
        m, r, s = C.c_float(), C.c_float(), C.c_float()
        check(load().psx_stats(_ptr(data), int(nsamps), int(first_samp), C.byref(m), C.byref(r),
                               C.byref(s), _stream()), "stats")
        return m.value, r.value, s.value

    @staticmethod
    def normalise(data: torch.Tensor, mean: float, std: float, size: int) -> None:
        check(load().psx_normalise(_ptr(data), mean, std, int(size), _stream()), "normalise")


normalise = stats.normalise


class SpectrumNormaliser:
    """The normalisation step of the search loop (pipeline_multi.cu:271,
    stats::normalise) as a transform: p = (p - mean*N) / (std*N)."""

    def __init__(self, mean: float, std: float, fft_size: int):
        self.mean = np.float32(np.float32(mean) * np.float32(fft_size))
        self.std = np.float32(np.float32(std) * np.float32(fft_size))

    def normalise(self, pspec: DevicePowerSpectrum) -> None:
        stats.normalise(pspec.data, float(self.mean), float(self.std), pspec.get_nbins())


class HarmonicFolder:
    """include/transforms/harmonicfolder.hpp:8-45."""

    def __init__(self, sums: HarmonicSums):
        self.sums = sums

    def fold(self, fold0: DevicePowerSpectrum) -> None:
        n = self.sums.size()
        ptrs = (C.c_void_p * max(1, n))(*[s.data.data_ptr() for s in self.sums.folds])
        check(load().psx_harmonic_sum(_ptr(fold0.data), ptrs, fold0.get_nbins(), n, _stream()),
              "HarmonicFolder::fold")


# --------------------------------------------------------------- candidates
class Candidate:
    """include/data_types/candidates.hpp:19-97 (the fields the search fills)."""
    __slots__ = ("dm", "dm_idx", "acc", "nh", "snr", "freq", "assoc")

    def __init__(self, dm=0.0, dm_idx=0, acc=0.0, nh=0, snr=0.0, freq=0.0):
        self.dm, self.dm_idx, self.acc = float(dm), int(dm_idx), float(acc)
        self.nh, self.snr, self.freq = int(nh), float(snr), float(freq)
        self.assoc: List["Candidate"] = []

    def append(self, other: "Candidate") -> None:
        self.assoc.append(other)

    def count_assoc(self) -> int:
        return sum(1 + a.count_assoc() for a in self.assoc)

    def pod(self) -> tuple:
        return (self.dm, self.dm_idx, self.acc, self.nh, self.snr, self.freq)

    def __repr__(self):
        return (f"Candidate(dm={self.dm:g}, acc={self.acc:g}, nh={self.nh}, "
                f"snr={self.snr:.4f}, freq={self.freq:.9g})")


class CandidateCollection:
    """candidates.hpp:99-149."""

    def __init__(self):
        self.cands: List[Candidate] = []

    def append(self, other) -> None:
        self.cands.extend(other.cands if isinstance(other, CandidateCollection) else other)

    def reset(self) -> None:
        self.cands.clear()


class SpectrumCandidates(CandidateCollection):
    """candidates.hpp:152-166."""

    def __init__(self, dm: float, dm_idx: int, acc: float):
        super().__init__()
        self.dm, self.dm_idx, self.acc = dm, dm_idx, acc

    def append_peaks(self, snrs, freqs, nh: int) -> None:
        for s, f in zip(snrs, freqs):
            self.cands.append(Candidate(self.dm, self.dm_idx, self.acc, nh, s, f))


class PeakFinder:
    """include/transforms/peakfinder.hpp:11-95."""

    def __init__(self, threshold: float, min_freq: float, max_freq: float, size: int,
                 min_gap: int = 30):
        _require_cuda()
        self.threshold = float(threshold)
        self.min_freq = float(min_freq)
        self.max_freq = float(max_freq)
        self.min_gap = int(min_gap)
        self.cap = max(1024, int(size))
        self.d_idx = torch.zeros(self.cap, dtype=torch.int32, device="cuda")
        self.d_val = torch.zeros(self.cap, dtype=torch.float32, device="cuda")

    def find_candidates(self, spec, cands: SpectrumCandidates) -> None:
        if isinstance(spec, HarmonicSums):
            for s in spec.folds:
                self.find_candidates(s, cands)
            return
        L = load()
        size = spec.get_nbins()
        start, end, factor = C.c_int(), C.c_int(), C.c_float()
        check(L.psx_peak_range(size, spec.get_bin_width(), spec.get_nh(), self.min_freq,
                               self.max_freq, C.byref(start), C.byref(end), C.byref(factor)),
              "peak_range")
        count = C.c_int()
        rc = L.psx_find_peaks(_ptr(spec.data), end.value, start.value, self.threshold,
                              _ptr(self.d_idx), _ptr(self.d_val), self.cap, C.byref(count),
                              _stream())
        if rc == _lib.PSX_ERR_OVERFLOW:
            self.cap = int(count.value * 1.25) + 1024
            self.d_idx = torch.zeros(self.cap, dtype=torch.int32, device="cuda")
            self.d_val = torch.zeros(self.cap, dtype=torch.float32, device="cuda")
            rc = L.psx_find_peaks(_ptr(spec.data), end.value, start.value, self.threshold,
                                  _ptr(self.d_idx), _ptr(self.d_val), self.cap, C.byref(count),
                                  _stream())
        check(rc, "find_peaks")
        n = count.value
        if n == 0:
            return
        idx = self.d_idx[:n].cpu().numpy()
        val = self.d_val[:n].cpu().numpy()
        pi = np.zeros(n, np.int32)
        ps = np.zeros(n, np.float32)
        npk = L.psx_identify_unique_peaks(idx.ctypes.data, val.ctypes.data, n, self.min_gap,
                                          pi.ctypes.data, ps.ctypes.data)
        freqs = (pi[:npk].astype(np.float32) * np.float32(factor.value)).astype(np.float32)
        cands.append_peaks(ps[:npk].tolist(), freqs.tolist(), spec.get_nh())


# --------------------------------------------------------------- distillers
def _to_pod(cands: Sequence[Candidate]):
    arr = (_CandPOD * max(1, len(cands)))()
    for i, c in enumerate(cands):
        arr[i] = _CandPOD(*c.pod())
    return arr


class _Distiller:
    kind = 0

    def __init__(self, tol: float, max_harm: float = 16.0, tobs: float = 0.0,
                 keep_related: bool = False, fractional: bool = True):
        self.tol, self.max_harm, self.tobs = tol, max_harm, tobs
        self.keep_related, self.fractional = keep_related, fractional

    def distill(self, cands: List[Candidate]) -> List[Candidate]:
        """distiller.hpp:30-56: sorts `cands` by S/N (in place, as the
        reference does) and returns the survivors."""
        n = len(cands)
        if n == 0:
            return []
        arr = _to_pod(cands)
        na = np.zeros(n, np.int32)
        keep = load().psx_distill(self.kind, arr, n, self.tol, self.max_harm, self.tobs,
                                  int(self.keep_related), int(self.fractional), na.ctypes.data)
        out = []
        for i in range(keep):
            a = arr[i]
            c = Candidate(a.dm, a.dm_idx, a.acc, a.nh, a.snr, a.freq)
            c.assoc = [Candidate()] * int(na[i])  # association count only
            out.append(c)
        return out


class HarmonicDistiller(_Distiller):
    """distiller.hpp:63-108."""
    kind = _lib.PSX_DISTILL_HARMONIC

    def __init__(self, tol: float, max_harm: float, keep_related: bool,
                 fractional_harms: bool = True):
        super().__init__(tol, max_harm, 0.0, keep_related, fractional_harms)


class AccelerationDistiller(_Distiller):
    """distiller.hpp:115-163."""
    kind = _lib.PSX_DISTILL_ACCEL

    def __init__(self, tobs: float, tolerance: float, keep_related: bool):
        super().__init__(tolerance, 16.0, tobs, keep_related, True)


class DMDistiller(_Distiller):
    """distiller.hpp:167-196."""
    kind = _lib.PSX_DISTILL_DM

    def __init__(self, tolerance: float, keep_related: bool):
        super().__init__(tolerance, 16.0, 0.0, keep_related, True)


class AccelerationPlan:
    """include/utils/utils.hpp:143-233 (all arithmetic in float, as there)."""

    def __init__(self, acc_lo, acc_hi, tol, pulse_width, nsamps, tsamp, cfreq, ch_bw):
        self.args = (float(acc_lo), float(acc_hi), float(tol), float(pulse_width), int(nsamps),
                     float(tsamp), float(cfreq), float(ch_bw))

    def generate_accel_list(self, dm: float, cdm: float) -> np.ndarray:
        L = load()
        n = C.c_size_t()
        check(L.psx_accel_list(*self.args, dm, cdm, None, 0, C.byref(n)), "accel_list")
        out = np.zeros(max(1, n.value), np.float32)
        check(L.psx_accel_list(*self.args, dm, cdm, out.ctypes.data, out.size, C.byref(n)),
              "accel_list")
        return out[:n.value].copy()
