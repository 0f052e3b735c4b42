"""After the DM loop: the reference's global distillation, scoring and output
files (src/pipeline_multi.cu:531-587), on candidate forests.

A forest is ``(nodes, sizes)``: candidate records (``search.CAND_DTYPE``)
in depth-first order and, per node, the size of the subtree it roots.  The
per-DM forests come from ``AccelSearch.search_block(..., per_dm="forest")``
(or ``psx_search_block`` with ``PSX_OUT_DM_FOREST``); ``finish`` runs the
DMDistiller and HarmonicDistiller with their association trees, the
CandidateScorer, the candidate limit, and writes ``candidates.peasoup`` and
``overview.xml`` as the reference does.  Everything here is host C++ in
libpeasoup_b200 reached through the C ABI.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from typing import Dict, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, load
from .search import CAND_DTYPE

SCORE_DTYPE = np.dtype([("is_physical", "<i4"), ("is_adjacent", "<i4"),
                        ("ddm_count_ratio", "<f4"), ("ddm_snr_ratio", "<f4"),
                        ("nassoc", "<i4")])


def roots(sizes) -> np.ndarray:
    """Start index of every top-level subtree."""
    out, i = [], 0
    while i < len(sizes):
        out.append(i)
        i += int(sizes[i])
    return np.asarray(out, np.int64)


def leaves(cands) -> tuple:
    """A forest of single-node trees."""
    a = np.ascontiguousarray(cands, CAND_DTYPE)
    return a, np.ones(a.size, np.int32)


def concat(forests) -> tuple:
    """Forests one after another (the reference appends the Workers' lists)."""
    fs = [f for f in forests if len(f[0])]
    if not fs:
        return np.zeros(0, CAND_DTYPE), np.zeros(0, np.int32)
    return (np.concatenate([np.ascontiguousarray(f[0], CAND_DTYPE) for f in fs]),
            np.concatenate([np.ascontiguousarray(f[1], np.int32) for f in fs]))


def distill_forest(kind: int, nodes, sizes, tol: float = 1e-4, max_harm: float = 16.0,
                   tobs: float = 0.0, keep_related: bool = True, fractional: bool = False):
    a = np.ascontiguousarray(nodes, CAND_DTYPE)
    sz = np.ascontiguousarray(sizes, np.int32)
    L = load()
    cap = max(16, 2 * a.size)
    while True:
        out = np.zeros(cap, CAND_DTYPE)
        osz = np.zeros(cap, np.int32)
        n, nr = C.c_size_t(), C.c_size_t()
        rc = L.psx_distill_forest(kind, a.ctypes.data, sz.ctypes.data, a.size, tol, max_harm, tobs,
                                  int(keep_related), int(fractional), out.ctypes.data,
                                  osz.ctypes.data, cap, C.byref(n), C.byref(nr))
        if rc == _lib.PSX_ERR_OVERFLOW:
            cap = n.value
            continue
        check(rc, "distill_forest")
        return out[:n.value].copy(), osz[:n.value].copy()


def score_forest(nodes, sizes, tsamp: float, cfreq_mhz: float, foff_mhz: float,
                 bw_mhz: float) -> np.ndarray:
    a = np.ascontiguousarray(nodes, CAND_DTYPE)
    sz = np.ascontiguousarray(sizes, np.int32)
    cap = max(1, len(roots(sz)))
    out = np.zeros(cap, SCORE_DTYPE)
    n = C.c_size_t()
    check(load().psx_score_forest(a.ctypes.data, sz.ctypes.data, a.size, tsamp, cfreq_mhz,
                                  foff_mhz, bw_mhz, out.ctypes.data, cap, C.byref(n)),
          "score_forest")
    return out[:n.value]


def limit(nodes, sizes, count: int):
    """The first `count` candidates with their trees (--limit)."""
    r = roots(sizes)
    if count >= len(r):
        return nodes, sizes
    end = int(r[count]) if count > 0 else 0
    return nodes[:end], sizes[:end]


def write_candidates(path: str, nodes, sizes) -> np.ndarray:
    """candidates.peasoup; returns each candidate's byte offset."""
    a = np.ascontiguousarray(nodes, CAND_DTYPE)
    sz = np.ascontiguousarray(sizes, np.int32)
    cap = max(1, len(roots(sz)))
    off = np.zeros(cap, np.int64)
    n = C.c_size_t()
    check(load().psx_write_candidates(path.encode(), a.ctypes.data, sz.ctypes.data, a.size,
                                      off.ctypes.data, cap, C.byref(n)), "write_candidates")
    return off[:n.value]


def _fmt(v) -> str:
    """A value as the reference's XML writer prints it (precision 15)."""
    if isinstance(v, (bool, np.bool_)):
        return "1" if v else "0"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return "%.15g" % float(v)
    return str(v)


class Overview:
    """overview.xml, section by section (OutputFileWriter)."""

    def __init__(self):
        self._h = C.c_void_p()
        check(load().psx_overview_create(C.byref(self._h)), "overview_create")

    def __del__(self):
        if getattr(self, "_h", None):
            load().psx_overview_destroy(self._h)
            self._h = None

    def section(self, name: str, items: Dict[str, object]):
        keys = [k.encode() for k in items]
        vals = [_fmt(v).encode() for v in items.values()]
        ka = (C.c_char_p * max(1, len(keys)))(*keys)
        va = (C.c_char_p * max(1, len(vals)))(*vals)
        check(load().psx_overview_add_section(self._h, name.encode(), ka, va, len(keys)),
              "overview_add_section")
        return self

    def misc_info(self, unix_time: Optional[int] = None):
        check(load().psx_overview_add_misc_info(self._h, int(time.time() if unix_time is None
                                                             else unix_time)), "overview_misc")
        return self

    def dm_list(self, dms):
        d = np.ascontiguousarray(dms, np.float32)
        check(load().psx_overview_add_dm_list(self._h, d.ctypes.data, d.size), "overview_dm_list")
        return self

    def acc_list(self, accs, cdm: float):
        a = np.ascontiguousarray(accs, np.float32)
        check(load().psx_overview_add_acc_list(self._h, a.ctypes.data, a.size, cdm),
              "overview_acc_list")
        return self

    def device_info(self, devices: Sequence[int]):
        import torch
        rt = C.c_int()
        dv = C.c_int()
        try:
            cudart = C.CDLL("libcudart.so")
            cudart.cudaRuntimeGetVersion(C.byref(rt))
            cudart.cudaDriverGetVersion(C.byref(dv))
        except OSError:
            pass
        props = [torch.cuda.get_device_properties(d) for d in devices]
        ids = np.asarray(devices, np.int32)
        names = (C.c_char_p * max(1, len(props)))(*[p.name.encode() for p in props])
        major = np.asarray([p.major for p in props], np.int32)
        minor = np.asarray([p.minor for p in props], np.int32)
        check(load().psx_overview_add_device_info(self._h, rt.value, dv.value, ids.ctypes.data,
                                                  names, major.ctypes.data, minor.ctypes.data,
                                                  len(props)), "overview_device_info")
        return self

    def candidates(self, nodes, sizes, scores, offsets):
        a = np.ascontiguousarray(nodes, CAND_DTYPE)
        sz = np.ascontiguousarray(sizes, np.int32)
        sc = np.ascontiguousarray(scores, SCORE_DTYPE)
        off = np.ascontiguousarray(offsets, np.int64)
        check(load().psx_overview_add_candidates(self._h, a.ctypes.data, sz.ctypes.data, a.size,
                                                 sc.ctypes.data, off.ctypes.data),
              "overview_add_candidates")
        return self

    def text(self) -> str:
        n = C.c_size_t()
        check(load().psx_overview_write(self._h, None, None, 0, C.byref(n)), "overview_write")
        buf = C.create_string_buffer(n.value + 1)
        check(load().psx_overview_write(self._h, None, buf, n.value + 1, C.byref(n)),
              "overview_write")
        return buf.value.decode("latin-1")

    def write(self, path: str):
        n = C.c_size_t()
        check(load().psx_overview_write(self._h, path.encode(), None, 0, C.byref(n)),
              "overview_write")


def finish(dm_forests, outdir: str, *, tsamp: float, cfreq_mhz: float, foff_mhz: float,
           bw_mhz: float, freq_tol: float = 1e-4, max_harm: float = 16.0,
           limit_count: int = 1000, dms=None, accs=None, cdm: float = 0.0,
           sections: Optional[Dict[str, Dict[str, object]]] = None, devices=None,
           timings: Optional[Dict[str, float]] = None):
    """src/pipeline_multi.cu:547-587 on the per-DM forests: DMDistiller and
    HarmonicDistiller (keep_related; harmonics not fractional), scores,
    --limit, then candidates.peasoup and overview.xml in `outdir`.  Returns
    (nodes, sizes, scores, byte offsets) of the written candidates."""
    nodes, sizes = concat(dm_forests)
    nodes, sizes = distill_forest(_lib.PSX_DISTILL_DM, nodes, sizes, tol=freq_tol,
                                  keep_related=True)
    nodes, sizes = distill_forest(_lib.PSX_DISTILL_HARMONIC, nodes, sizes, tol=freq_tol,
                                  max_harm=max_harm, keep_related=True, fractional=False)
    scores = score_forest(nodes, sizes, tsamp, cfreq_mhz, foff_mhz, bw_mhz)
    nodes, sizes = limit(nodes, sizes, limit_count)
    scores = scores[:len(roots(sizes))]
    os.makedirs(outdir, exist_ok=True)
    offsets = write_candidates(os.path.join(outdir, "candidates.peasoup"), nodes, sizes)
    ov = Overview().misc_info()
    for name, items in (sections or {}).items():
        ov.section(name, items)
    if dms is not None:
        ov.dm_list(dms)
    if accs is not None:
        ov.acc_list(accs, cdm)
    if devices:
        ov.device_info(devices)
    ov.candidates(nodes, sizes, scores, offsets)
    if timings:
        ov.section("execution_times", timings)
    ov.write(os.path.join(outdir, "overview.xml"))
    return nodes, sizes, scores, offsets
