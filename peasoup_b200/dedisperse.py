"""Dedispersion into device-resident series: the reference's Dedisperser and
DispersionTrials (include/transforms/dedisperser.hpp:13-188,
include/data_types/timeseries.hpp:465-596) over psx_dedisp_* of
libpeasoup_b200.so.

The reference dedisperses on the GPU through dedisp, copies every series to
the host (DispersionTrials) and copies them back one at a time in each
Worker.  Here the dedispersed block stays on the device as a (ndm, pitch)
float32 CUDA tensor whose rows feed AccelSearch.search_block directly;
DispersionTrials.to_host() gives the reference's host block when wanted.
"""
from __future__ import annotations

import ctypes as C
import sys
from typing import List, Optional, Sequence, Union

import numpy as np
import torch

from . import _lib
from ._lib import PsxError, check, load
from .sigproc import SigprocFilterbank

__all__ = ["Dedisperser", "DispersionTrials"]


def _stream() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class DispersionTrials:
    """ndm dedispersed series of nsamps samples on the device, one row per
    DM trial (rows `pitch` floats apart)."""

    def __init__(self, tsamp: float):
        self.tsamp = float(tsamp)
        self.nsamps = 0
        self.dm_list = np.zeros(0, np.float32)
        self.data: Optional[torch.Tensor] = None

    def resize(self, out_nsamps: int, dm_list: Sequence[float]) -> None:
        self.dm_list = np.ascontiguousarray(dm_list, np.float32)
        self.nsamps = int(out_nsamps)
        pitch = (self.nsamps + 3) // 4 * 4
        if (self.data is None or self.data.shape[0] != len(self.dm_list)
                or self.data.shape[1] != pitch):
            self.data = torch.empty((len(self.dm_list), pitch), dtype=torch.float32,
                                    device="cuda")

    def __len__(self) -> int:
        return len(self.dm_list)

    def __getitem__(self, idx: int) -> torch.Tensor:
        return self.data[idx, :self.nsamps]

    def rows(self) -> List[torch.Tensor]:
        return [self[i] for i in range(len(self))]

    def get_dm_list(self) -> np.ndarray:
        return self.dm_list

    def get_nsamps(self) -> int:
        return self.nsamps

    def get_tsamp(self) -> float:
        return self.tsamp

    def to_host(self) -> np.ndarray:
        return self.data[:, :self.nsamps].cpu().numpy()


class Dedisperser:
    """Dedisperser(filterbank) with the reference's methods; the plan holds
    the channel delays and DM list, and its device scratch."""

    def __init__(self, filterbank: SigprocFilterbank, num_gpus: int = 1):
        if not torch.cuda.is_available():
            raise PsxError(_lib.PSX_ERR_CUDA, "Dedisperser", "no CUDA device (no CPU fallback)")
        self.filterbank = filterbank
        self.num_gpus = num_gpus
        self._plan = C.c_void_p()
        check(load().psx_dedisp_create(filterbank.get_nchans(), filterbank.get_tsamp(),
                                       filterbank.get_fch1(), filterbank.get_foff(),
                                       C.byref(self._plan)), "dedisp_create")
        self.killmask = np.ones(filterbank.get_nchans(), np.int32)
        self._pinned: Optional[torch.Tensor] = None

    def close(self) -> None:
        if self._plan:
            load().psx_dedisp_destroy(self._plan)
            self._plan = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # DM list (dedisperser.hpp:43-71)
    def set_dm_list(self, dm_list: Sequence[float]) -> None:
        a = np.ascontiguousarray(dm_list, np.float32)
        check(load().psx_dedisp_set_dm_list(self._plan, a.ctypes.data, a.size), "set_dm_list")

    def generate_dm_list(self, dm_start: float, dm_end: float, width: float,
                         tolerance: float) -> None:
        check(load().psx_dedisp_generate_dm_list(self._plan, dm_start, dm_end, width,
                                                 tolerance), "generate_dm_list")

    def get_dm_list(self) -> np.ndarray:
        L = load()
        n = L.psx_dedisp_get_dm_count(self._plan)
        out = np.zeros(max(1, n), np.float32)
        if n:
            check(L.psx_dedisp_get_dm_list(self._plan, out.ctypes.data, n), "get_dm_list")
        return out[:n]

    def get_delay_table(self) -> np.ndarray:
        out = np.zeros(self.filterbank.get_nchans(), np.float32)
        check(load().psx_dedisp_get_delay_table(self._plan, out.ctypes.data), "delay_table")
        return out

    def get_max_delay(self) -> int:
        return int(load().psx_dedisp_get_max_delay(self._plan))

    # killmask (dedisperser.hpp:73-110)
    def set_killmask(self, killmask: Union[str, Sequence[int]]) -> None:
        """A list of nchans flags (0 drops the channel), or a file of one
        integer per line, read for at most nchans lines; a file of the wrong
        length leaves every channel in, with a warning, as the reference
        does."""
        nchans = self.filterbank.get_nchans()
        if isinstance(killmask, str):
            vals = []
            with open(killmask, "rb") as f:
                for line in f:
                    if len(vals) >= nchans:
                        break
                    s = line.decode(errors="replace").strip()
                    try:
                        vals.append(int(s.split()[0]) if s else 0)
                    except ValueError:
                        vals.append(0)
            if len(vals) != nchans:
                sys.stderr.write("WARNING: killmask is not the same size as nchans\n"
                                 f"{len(vals)} != {nchans}\n")
                vals = [1] * nchans
            killmask = vals
        km = np.ascontiguousarray(killmask, np.int32)
        if km.size != nchans:
            raise PsxError(_lib.PSX_ERR_INVALID, "set_killmask", "killmask size != nchans")
        check(load().psx_dedisp_set_killmask(self._plan, km.ctypes.data), "set_killmask")
        self.killmask = km

    # execution
    def execute(self, rows: Union[np.ndarray, torch.Tensor], nsamps: int, out: torch.Tensor,
                raw: bool = False) -> None:
        """Dedisperse nsamps packed rows (host array or CUDA uint8 tensor)
        into the rows of `out` (ndm, pitch) float32 CUDA tensor."""
        L = load()
        flags = _lib.PSX_DEDISP_RAW if raw else 0
        nbits = self.filterbank.get_nbits()
        if not (out.is_cuda and out.dtype == torch.float32 and out.is_contiguous()):
            raise PsxError(_lib.PSX_ERR_INVALID, "execute", "out must be a contiguous CUDA "
                           "float32 tensor")
        if isinstance(rows, torch.Tensor) and rows.is_cuda:
            check(L.psx_dedisp_execute(self._plan, nsamps, C.c_void_p(rows.data_ptr()), nbits,
                                       C.c_void_p(out.data_ptr()), out.shape[1], flags,
                                       _stream()), "dedisp_execute")
        else:
            if isinstance(rows, torch.Tensor):
                ptr, keep = rows.data_ptr(), rows
            else:
                keep = np.ascontiguousarray(rows, np.uint8)
                ptr = keep.ctypes.data
            check(L.psx_dedisp_execute_host(self._plan, nsamps, C.c_void_p(ptr), nbits,
                                            C.c_void_p(out.data_ptr()), out.shape[1], flags,
                                            _stream()), "dedisp_execute_host")
            del keep

    def dedisperse(self, trials: Optional[DispersionTrials] = None,
                   input_start_sample: Optional[int] = None,
                   input_end_sample: Optional[int] = None, gulp: int = 0,
                   raw: bool = False) -> DispersionTrials:
        """Dedisperses samples [start, end) of the filterbank (default: its
        segment) into `trials`: nsamps - max_delay samples per DM trial, as
        Dedisperser::dedisperse (dedisperser.hpp:112-186).  The file is read
        in pieces of `gulp` samples (any value; the whole span by default)
        into pinned host memory and dedispersed in one pass on the device."""
        fb = self.filterbank
        start = fb.get_start_sample() if input_start_sample is None else int(input_start_sample)
        end = fb.get_end_sample() if input_end_sample is None else int(input_end_sample)
        nsamps = end - start
        md = self.get_max_delay()
        if nsamps <= md:
            raise PsxError(_lib.PSX_ERR_INVALID, "dedisperse",
                           f"{nsamps} samples do not exceed the maximum delay {md}")
        rb = fb.row_bytes()
        if self._pinned is None or self._pinned.numel() < nsamps * rb:
            self._pinned = torch.empty(nsamps * rb, dtype=torch.uint8, pin_memory=True)
        else:
            torch.cuda.current_stream().synchronize()  # earlier copies from the buffer
        host = self._pinned.numpy()
        step = nsamps if gulp <= 0 else int(gulp)
        pos = 0
        while pos < nsamps:
            n = min(step, nsamps - pos)
            got = fb.load_gulp(start + pos, n, out=host[pos * rb:(pos + n) * rb])
            if got == 0:
                raise PsxError(_lib.PSX_ERR_IO, "dedisperse",
                               "Failed to read data during dedispersion, 0 samples read.")
            pos += got
        if trials is None:
            trials = DispersionTrials(fb.get_tsamp())
        trials.resize(nsamps - md, self.get_dm_list())
        self.execute(self._pinned, nsamps, trials.data, raw=raw)
        return trials
