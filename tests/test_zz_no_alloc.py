"""psx_find_peaks_noalloc, the peak finder that allocates no device memory.

Its per-tile counts live in an array compiled into the library instead of
memory from cudaMallocAsync.  The GPU test checks it against
psx_find_peaks (bit-exact: the compaction copies indices and values) on
two calls in a row, the second over fewer tiles than the first, so that
counts the first call left in the shared array would show up as wrong
offsets.  This file is collected last so that it runs both alone and after
every other test in one process.
"""
import ctypes as C

import numpy as np
import pytest

PSX_OK, PSX_ERR_INVALID, PSX_ERR_OVERFLOW = 0, 1, 5
MAX_BINS = 1 << 28          # the static scratch's limit on n - start


def _find(fn, torch, spec, n, start, thresh, cap):
    idx = torch.full((max(cap, 1),), -1, dtype=torch.int32, device="cuda")
    val = torch.full((max(cap, 1),), np.nan, dtype=torch.float32, device="cuda")
    count = C.c_int(-7)
    rc = fn(C.c_void_p(spec.data_ptr()), n, start, thresh, C.c_void_p(idx.data_ptr()),
            C.c_void_p(val.data_ptr()), cap, C.byref(count), None)
    torch.cuda.synchronize()
    k = min(count.value, cap)
    return rc, count.value, idx[:k].cpu().numpy(), val[:k].cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_find_peaks_on_consecutive_calls(psx, cuda):
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(29)
    cases = [
        # (bins, start, threshold): the second call covers far fewer tiles
        ((1 << 22) + 37, 5000, 3.5),
        (70001, 13, 2.8),
    ]
    specs = []
    for n, start, _ in cases:
        spec = torch.randn(n, device="cuda", generator=g)
        spec[start + 1::9973] = 50.0            # a regular train of strong bins
        specs.append(spec)
    wants = [_find(psx.psx_find_peaks, torch, s, n, start, t, 1 << 14)
             for s, (n, start, t) in zip(specs, cases)]
    # the two calls of the no-allocation entry point follow one another
    gots = [_find(psx.psx_find_peaks_noalloc, torch, s, n, start, t, 1 << 14)
            for s, (n, start, t) in zip(specs, cases)]
    for spec, (n, start, thresh), want, got in zip(specs, cases, wants, gots):
        assert want[0] == PSX_OK and got[0] == PSX_OK, psx.psx_last_error()
        assert got[1] == want[1] > 100
        assert np.array_equal(got[2], want[2])
        assert np.array_equal(got[3], want[3])
        # against the definition, on the host
        h = spec.cpu().numpy()
        sel = np.flatnonzero(h[start:] > thresh) + start
        assert np.array_equal(got[2], sel) and np.array_equal(got[3], h[sel])

    # a buffer too small reports the full count, as psx_find_peaks does
    rc_w, cnt_w, iw, vw = _find(psx.psx_find_peaks, torch, spec, n, 0, thresh, 50)
    rc_g, cnt_g, ig, vg = _find(psx.psx_find_peaks_noalloc, torch, spec, n, 0, thresh, 50)
    assert rc_w == rc_g == PSX_ERR_OVERFLOW and cnt_w == cnt_g > 50
    assert np.array_equal(ig, iw) and np.array_equal(vg, vw)


def test_noalloc_rejects_more_bins_than_its_scratch_holds(psx):
    """The size check comes before any CUDA call, so this runs without a
    device; the pointer is never dereferenced."""
    host = np.zeros(4, np.float32)
    p = C.c_void_p(host.ctypes.data)
    count = C.c_int(-1)
    n = MAX_BINS + 1
    rc = psx.psx_find_peaks_noalloc(p, n, 0, 1.0, p, p, 4, C.byref(count), None)
    assert rc == PSX_ERR_INVALID
    assert b"static scratch" in psx.psx_last_error()
    assert count.value == 0
