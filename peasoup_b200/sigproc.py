"""SIGPROC filterbank input: the reference's SigprocHeader, read_header and
SigprocFilterbank (include/data_types/header.hpp:171-212, 339-403;
include/data_types/filterbank.hpp:25-328) and the DM list file reader
(getFileContent, src/pipeline_multi.cu:313-337), over the C ABI of
libpeasoup_b200.so.

Metadata keeps the reference's types: the Filterbank members tsamp, fch1
and foff are float, nchans and nbits integers (filterbank.hpp:34-45).
"""
from __future__ import annotations

import ctypes as C
import sys
from typing import Optional

import numpy as np

from . import _lib
from ._lib import SigprocHeader, check, load

__all__ = ["SigprocHeader", "read_header", "write_header", "write_filterbank",
           "SigprocFilterbank", "read_dm_file", "prev_power_of_two", "write_timeseries"]


def read_header(path: str) -> SigprocHeader:
    h = SigprocHeader()
    check(load().psx_sigproc_read_header(path.encode(), C.byref(h)), "sigproc_read_header")
    return h


def write_header(path: str, h: SigprocHeader) -> int:
    """Writes a header to a new file; returns its size in bytes."""
    n = C.c_size_t()
    check(load().psx_sigproc_write_header(path.encode(), C.byref(h), C.byref(n)),
          "sigproc_write_header")
    return n.value


def make_header(**fields) -> SigprocHeader:
    h = SigprocHeader()
    for k, v in fields.items():
        if k in ("source_name", "rawdatafile"):
            v = v.encode() if isinstance(v, str) else v
        setattr(h, k, v)
    return h


def write_filterbank(path: str, rows: np.ndarray, **fields) -> SigprocHeader:
    """A SIGPROC file of packed sample rows (uint8, one row per sample) with
    a header made of `fields`; returns the header as read back."""
    rows = np.ascontiguousarray(rows, np.uint8)
    write_header(path, make_header(**fields))
    with open(path, "ab") as f:
        f.write(rows.tobytes())
    return read_header(path)


def pack_samples(values: np.ndarray, nbits: int) -> np.ndarray:
    """(nsamps, nchans) unsigned samples -> packed SIGPROC rows: below 8
    bits the first channel in the least significant bits of its byte,
    16-bit samples little-endian."""
    v = np.asarray(values)
    ns, nc = v.shape
    if nbits == 8:
        return v.astype(np.uint8)
    if nbits == 16:
        return v.astype("<u2").view(np.uint8).reshape(ns, nc * 2)
    per = 8 // nbits
    if nc % per:
        raise ValueError("channels do not fill whole bytes")
    v = v.astype(np.uint8).reshape(ns, nc // per, per)
    out = np.zeros((ns, nc // per), np.uint8)
    for k in range(per):
        out |= (v[:, :, k] & ((1 << nbits) - 1)) << (k * nbits)
    return out


def prev_power_of_two(val: int) -> int:
    """Utils::prev_power_of_two (include/utils/utils.hpp:15-21)."""
    n = 1
    while n * 2 <= val:
        n *= 2
    return n


def read_dm_file(path: str) -> np.ndarray:
    """One DM per line; an empty line repeats the previous value."""
    L = load()
    n = C.c_size_t()
    rc = L.psx_read_dm_file(path.encode(), None, 0, C.byref(n))
    if rc not in (_lib.PSX_OK, _lib.PSX_ERR_OVERFLOW):
        check(rc, "read_dm_file")
    out = np.zeros(max(1, n.value), np.float32)
    check(L.psx_read_dm_file(path.encode(), out.ctypes.data, out.size, C.byref(n)),
          "read_dm_file")
    return out[:n.value]


class SigprocFilterbank:
    """A segment [start, end) of a SIGPROC file (filterbank.hpp:248-361).
    A segment of 0 samples, or one past the end, runs to the end of the
    file with a warning; a start past the end raises."""

    def __init__(self, filename: str, segment_start_sample: int = 0,
                 segment_nsamples: int = 0):
        self.filename = filename
        self._header = read_header(filename)
        h = self._header
        self.total_nsamps = int(h.nsamples)
        self.nchans = int(h.nchans)
        self.nbits = int(h.nbits)
        self.tsamp = float(np.float32(h.tsamp))
        self.fch1 = float(np.float32(h.fch1))
        self.foff = float(np.float32(h.foff))
        self.start_sample = int(segment_start_sample)
        if self.start_sample > self.total_nsamps:
            raise _lib.PsxError(_lib.PSX_ERR_INVALID, "SigprocFilterbank",
                                "Invalid start sample provided.")
        if segment_nsamples == 0 or self.start_sample + segment_nsamples > self.total_nsamps:
            sys.stderr.write("Warning: Requested segment exceeds total samples available in "
                             "filterbank. Adjusting to last available sample.\n")
            self.end_sample = self.total_nsamps
        else:
            self.end_sample = self.start_sample + int(segment_nsamples)
        self.effective_nsamps = self.end_sample - self.start_sample
        self.size = 0  # transform length, set by the caller for the pepoch
        self.data: Optional[np.ndarray] = None

    # Filterbank getters (filterbank.hpp:93-205)
    def get_tsamp(self) -> float: return self.tsamp
    def get_foff(self) -> float: return self.foff
    def get_fch1(self) -> float: return self.fch1
    def get_nchans(self) -> int: return self.nchans
    def get_nbits(self) -> int: return self.nbits
    def get_total_nsamps(self) -> int: return self.total_nsamps
    def get_start_sample(self) -> int: return self.start_sample
    def get_end_sample(self) -> int: return self.end_sample
    def get_effective_nsamps(self) -> int: return self.effective_nsamps
    def get_header(self) -> SigprocHeader: return self._header
    def get_data(self) -> Optional[np.ndarray]: return self.data

    def row_bytes(self) -> int:
        return self.nchans * self.nbits // 8

    def get_cfreq(self) -> float:
        """Centre frequency in MHz, in float as the reference computes it
        (filterbank.hpp:208-214)."""
        f, o, n = np.float32(self.fch1), np.float32(self.foff), np.float32(self.nchans)
        half = np.float32(o * n) / np.float32(2)
        return float(np.float32(f + half) if o < 0 else np.float32(f - half))

    def get_segment_pepoch(self) -> float:
        """MJD at the middle of the searched span (filterbank.hpp:336-343)."""
        ts = np.float32(self.tsamp)
        start_time = float(np.float32(self.start_sample) * ts) / 86400.0
        end_time = float(np.float32(self.size) * ts) / 86400.0
        return (self._header.tstart + start_time) + 0.5 * end_time

    def load_gulp(self, gulp_start_sample: int, gulp_nsamples: int,
                  out: Optional[np.ndarray] = None) -> int:
        """Reads packed rows into self.data (or `out`); returns rows read."""
        rb = self.row_bytes()
        buf = out if out is not None else np.empty(gulp_nsamples * rb, np.uint8)
        n = C.c_size_t()
        check(load().psx_sigproc_read(self.filename.encode(), C.byref(self._header),
                                      gulp_start_sample, gulp_nsamples, buf.ctypes.data,
                                      C.byref(n)), "sigproc_read")
        self.data = buf[:n.value * rb]
        return n.value


def _sexagesimal(value: float, signed: bool) -> str:
    """A SIGPROC angle (hhmmss.s / ddmmss.s packed in a double) as
    hh:mm:ss.ss, as the reference prints it (src/utils.cpp:14-74): the
    seconds get two decimals and no zero padding."""
    sign = -1 if value < 0 else 1
    a = abs(value)
    first = int(a / 1e4)
    second = int((a - first * 1e4) / 1e2)
    third = a - first * 1e4 - second * 1e2
    s = "%02d:%02d:%.2f" % (first, second, third)
    return ("-" + s) if (signed and sign < 0) else s


def write_timeseries(outdir: str, stem: str, series: np.ndarray, dm: float,
                     header: SigprocHeader) -> str:
    """One dedispersed series as `<outdir>/<stem>_DM<dm>.dat` (float32, an
    even number of samples) and its PRESTO-style `.inf`, as the reference's
    time-series dump writes them (DispersionTrials::write_timeseries_to_file,
    include/data_types/timeseries.hpp:520-594).  Returns the file prefix."""
    import os
    import pwd
    prefix = "%s/%s_DM%09.3f" % (outdir, stem, float(np.float32(dm)))
    x = np.ascontiguousarray(series, np.float32)
    n = x.size - (x.size % 2)
    x[:n].tofile(prefix + ".dat")
    h = header
    nchans = int(h.nchans)
    bw = float(h.foff) * nchans
    lowest = float(h.fch1) + float(h.foff) * (nchans - 1) if h.foff < 0 else float(h.fch1)
    try:
        login = pwd.getpwuid(os.getuid()).pw_name
    except KeyError:
        login = str(os.getuid())
    lines = [
        " Data file name without suffix          =  %s" % prefix,
        " Telescope used                         =  %d" % h.telescope_id,
        " Instrument used                        =  %d" % h.machine_id,
        " Object being observed                  =  %s" % h.source_name.decode(errors="replace"),
        " J2000 Right Ascension (hh:mm:ss.ssss)  =  %s" % _sexagesimal(h.src_raj, False),
        " J2000 Declination     (dd:mm:ss.ssss)  =  %s" % _sexagesimal(h.src_dej, True),
        " Data observed by                       =  pulsar_astronomer",
        " Epoch of observation (MJD)             =  %.15f" % h.tstart,
        " Barycentered?           (1=yes, 0=no)  =  0",
        " Number of bins in the time series      =  %d" % n,
        " Width of each time series bin (sec)    =  %.15f" % h.tsamp,
        " Any breaks in the data? (1 yes, 0 no)  =  0",
        " Type of observation (EM band)          =  Radio",
        " Beam diameter (arcsec)                 =  3600",
        " Dispersion measure (cm-3 pc)           =  %.15f" % float(np.float32(dm)),
        " Central freq of low channel (Mhz)      =  %.15f" % lowest,
        " Total bandwidth (Mhz)                  =  %.6f" % abs(bw),
        " Number of channels                     =  %d" % nchans,
        " Channel bandwidth (Mhz)                =  %.6f" % abs(bw),
        " Data analyzed by                       =  %s" % login,
        " Any additional notes:",
        "    File written by Peasoup pulsar search package",
    ]
    with open(prefix + ".inf", "w") as f:
        f.write("\n".join(lines) + "\n")
    return prefix
