"""psx_harmonic_peaks, the fused harmonic-sum + threshold + compaction
kernel on its own: its records equal the reference-order folds of
psx_harmonic_sum thresholded bin by bin (values bit for bit); a wait that
runs out (a test flag that stages nothing) fails the call with a status,
quickly, and leaves the context usable."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NBINS, ROWS, NH, THRESH = (1 << 16) + 1, 3, 4, 4.0


def _case(torch):
    g = torch.Generator(device="cuda").manual_seed(17)
    pitch = (NBINS + 63) // 64 * 64
    spec = torch.zeros((ROWS, pitch), device="cuda")
    spec[:, :NBINS] = torch.randn((ROWS, NBINS), device="cuda", generator=g).abs() * 1.3
    spec[:, 5000:5003] += 6.0   # a strong line and its harmonics
    spec[:, 10001] += 5.0
    start = np.array([40 << h for h in range(NH + 1)], np.int32)
    end = np.array([NBINS - 17 * (h + 1) for h in range(NH + 1)], np.int32)
    return spec, pitch, start, end


def _call(psx, spec, pitch, start, end, rec, cap, limit=0, flags=0):
    n = C.c_size_t()
    rc = psx.psx_harmonic_peaks(C.c_void_p(spec.data_ptr()), pitch, NBINS, ROWS, NH,
                                start.ctypes.data_as(C.c_void_p), end.ctypes.data_as(C.c_void_p),
                                THRESH, C.c_void_p(rec.data_ptr()), cap, C.byref(n), limit, flags,
                                None)
    return rc, n.value


def _expected(psx, torch, spec, start, end):
    """Folds by psx_harmonic_sum (the reference's order and scales), then
    every bin in range above the threshold."""
    want = set()
    for r in range(ROWS):
        row = spec[r, :NBINS].contiguous()
        folds = [torch.empty(NBINS, device="cuda") for _ in range(NH)]
        ptrs = (C.c_void_p * NH)(*[f.data_ptr() for f in folds])
        assert psx.psx_harmonic_sum(C.c_void_p(row.data_ptr()), ptrs, NBINS, NH, None) == 0
        torch.cuda.synchronize()
        for h, v in enumerate([row] + folds):
            a = v.cpu().numpy()
            idx = np.arange(start[h], end[h])
            sel = idx[a[start[h]:end[h]] > THRESH]
            for i in sel:
                want.add((r, h, int(i), int(np.float32(a[i]).view(np.int32))))
    return want


def test_records_equal_reference_folds(psx, cuda):
    torch = cuda
    spec, pitch, start, end = _case(torch)
    rec = torch.zeros((1 << 18, 4), dtype=torch.int32, device="cuda")
    rc, n = _call(psx, spec, pitch, start, end, rec, rec.shape[0])
    assert rc == 0, psx.psx_last_error()
    got = {tuple(int(v) for v in row) for row in rec[:n].cpu().numpy()}
    assert len(got) == n > 100
    assert got == _expected(psx, torch, spec, start, end)
    # a buffer too small reports the need
    small = torch.zeros((16, 4), dtype=torch.int32, device="cuda")
    rc, n2 = _call(psx, spec, pitch, start, end, small, 16)
    from peasoup_b200 import _lib
    assert rc == _lib.PSX_ERR_OVERFLOW and n2 == n


def test_wait_that_runs_out_fails_cleanly(psx, cuda):
    import time
    torch = cuda
    from peasoup_b200 import _lib
    spec, pitch, start, end = _case(torch)
    rec = torch.zeros((1 << 18, 4), dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    rc, n = _call(psx, spec, pitch, start, end, rec, rec.shape[0], limit=4096, flags=1)
    dt = time.perf_counter() - t0
    assert rc == _lib.PSX_ERR_CUDA and b"ran out" in psx.psx_last_error()
    assert dt < 10.0
    # the context is still usable: the same call without the flag succeeds
    rc, n = _call(psx, spec, pitch, start, end, rec, rec.shape[0])
    assert rc == 0 and n > 100
