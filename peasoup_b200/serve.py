"""The served loop from Python: a thin owner of a ``psx_server`` (C++, in
libpeasoup_b200) plus the request stream of the served benchmark.

``Server.submit`` queues a segmented search (a block of dedispersed series
of one transform length, its DM values and search parameters); the
server admits requests first in, first out, as worker slots and device
memory free up, and runs admitted requests concurrently on their own
search instances and CUDA streams.  ``Server.wait`` returns the per-DM
acceleration-distilled candidates and the request's timestamps.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import RequestStats, ServerConfig, check, load
from .search import CAND_DTYPE, SearchParams


POLICIES = {"least_work": _lib.PSX_SERVE_LEAST_WORK, "even": _lib.PSX_SERVE_EVEN,
            "exclusive": _lib.PSX_SERVE_EXCLUSIVE}


class Server:
    """One served loop on the current CUDA device."""

    def __init__(self, hbm_budget_bytes: int, max_active: int = 4, max_queue: int = 4096,
                 device: Optional[int] = None, policy: str = "exclusive"):
        """policy: "exclusive" (one request on the device at a time, the
        pending one with the least work next; measured best on the served
        workload), "least_work" (up to max_active requests at once, the one
        with the least work at the device's greatest stream priority) or
        "even" (up to max_active at once, no hint)."""
        if device is None:
            import torch
            device = torch.cuda.current_device()
        if policy not in POLICIES:
            raise ValueError("policy: " + ", ".join(POLICIES))
        cfg = ServerConfig(device=int(device), hbm_budget=int(hbm_budget_bytes),
                           max_active=int(max_active), max_queue=int(max_queue),
                           policy=POLICIES[policy])
        self._h = C.c_void_p()
        check(load().psx_server_create(C.byref(cfg), C.byref(self._h)), "server_create")
        self._keep = {}

    def close(self) -> None:
        if self._h:
            load().psx_server_destroy(self._h)
            self._h = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self) -> float:
        return float(load().psx_server_clock(self._h))

    def status(self) -> dict:
        used, act, pend, pool = C.c_size_t(), C.c_int(), C.c_int(), C.c_int()
        check(load().psx_server_status(self._h, C.byref(used), C.byref(act), C.byref(pend),
                                       C.byref(pool)), "server_status")
        return {"used_bytes": used.value, "active": act.value, "pending": pend.value,
                "pooled": pool.value}

    def submit(self, params: SearchParams, series, dms, dm_idx=None) -> int:
        """series: [ndm, nsamps] float32 torch CUDA tensor (stays on the
        device) or host array; it is kept alive until the result is taken."""
        ndm = len(dms)
        try:
            import torch
            is_dev = isinstance(series, torch.Tensor) and series.is_cuda
        except ImportError:
            is_dev = False
        if is_dev:
            t = series.contiguous()
            ptrs = (C.c_void_p * ndm)(*[t[d].data_ptr() for d in range(ndm)])
            nsamps = int(t.shape[1])
            hold = t
        else:
            a = np.ascontiguousarray(series, np.float32)
            ptrs = (C.c_void_p * ndm)(*[a[d].ctypes.data for d in range(ndm)])
            nsamps = int(a.shape[1])
            hold = a
        cfg, keep = params.to_c()
        d = np.ascontiguousarray(dms, np.float32)
        di = None if dm_idx is None else np.ascontiguousarray(dm_idx, np.int32)
        ticket = C.c_longlong()
        check(load().psx_server_submit(
            self._h, C.byref(cfg), ptrs, nsamps, int(is_dev), d.ctypes.data_as(C.c_void_p),
            None if di is None else di.ctypes.data_as(C.c_void_p), ndm, C.byref(ticket)),
            "server_submit")
        self._keep[ticket.value] = (hold, ptrs, keep, d, di)
        return ticket.value

    def wait(self, ticket: int, timeout: Optional[float] = None):
        """(candidates, nassoc, dm position, stats dict) of a request."""
        cap = 1 << 14
        st = RequestStats()
        while True:
            out = np.zeros(cap, CAND_DTYPE)
            na = np.zeros(cap, np.int32)
            dm = np.zeros(cap, np.int32)
            n = C.c_size_t()
            rc = load().psx_server_wait(self._h, ticket, -1.0 if timeout is None else timeout,
                                        out.ctypes.data_as(C.c_void_p),
                                        na.ctypes.data_as(C.c_void_p),
                                        dm.ctypes.data_as(C.c_void_p), cap, C.byref(n),
                                        C.byref(st))
            if rc == _lib.PSX_ERR_OVERFLOW:
                cap = n.value
                continue
            if rc != _lib.PSX_ERR_BUSY:
                self._keep.pop(ticket, None)
            check(rc, "server_wait")
            k = n.value
            stats = {f: getattr(st, f) for f, _ in RequestStats._fields_}
            return out[:k].copy(), na[:k].copy(), dm[:k].copy(), stats


# ------------------------------------------------------------ request stream
@dataclass
class ServedRequest:
    arrival: float          # seconds after the start of the stream
    fft_size: int
    ndm: int                # DM trials searched (after any bound)
    ndm_drawn: int          # DM trials drawn from the distribution
    acc_half: float         # m/s^2
    nharmonics: int
    tsamp: float = 64e-6


SERVED_SIZES = (1 << 20, 1 << 21, 3 << 20, 1 << 22, 3 << 21, 1 << 23, 1 << 24, 1 << 25)


def served_stream(n: int, seed: int = 1, rate: float = 4.0, trial_budget: Optional[int] = None,
                  max_ndm: Optional[int] = None) -> List[ServedRequest]:
    """The served workload's request stream: Poisson arrivals at `rate`
    per second (seeded), fft_size uniform over SERVED_SIZES, DM-trial count
    log-uniform over 16..512, acceleration half-range uniform over
    10..300 m/s^2, folds uniform over {3, 4, 5}.  `trial_budget` bounds a
    request's work: its DM count is cut so that DM count x (DM-0
    acceleration trials) x fft_size / 2^23 stays within the budget (the
    offered load far exceeds one GPU otherwise); `max_ndm` caps it too."""
    from .transforms import AccelerationPlan
    from . import synth
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        N = int(SERVED_SIZES[rng.integers(len(SERVED_SIZES))])
        ndm = int(round(math.exp(rng.uniform(math.log(16), math.log(512)))))
        acc = float(rng.uniform(10.0, 300.0))
        nh = int(rng.integers(3, 6))
        k = ndm
        if trial_budget is not None:
            ap = AccelerationPlan(-acc, acc, 1.10, 64e-6, N, 64e-6, synth.CFREQ_HZ,
                                  synth.CH_BW_HZ)
            ntr = len(ap.generate_accel_list(0.0, 0.0))
            unit = ntr * N / float(1 << 23)
            k = max(1, min(ndm, int(trial_budget // max(unit, 1e-9))))
        if max_ndm is not None:
            k = min(k, max_ndm)
        out.append(ServedRequest(arrival=t, fft_size=N, ndm=k, ndm_drawn=ndm, acc_half=acc,
                                 nharmonics=nh))
    return out


def request_params(r: ServedRequest) -> SearchParams:
    from . import synth
    return SearchParams(fft_size=r.fft_size, tsamp=r.tsamp, acc_lo=-r.acc_half,
                        acc_hi=r.acc_half, nharmonics=r.nharmonics, cfreq_hz=synth.CFREQ_HZ,
                        ch_bw_hz=synth.CH_BW_HZ, min_snr=7.0)
