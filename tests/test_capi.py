"""The C-ABI library on the CPU: it loads, exports every entry point the
public header declares, and its host logic (acceleration plan, peak
ranges, clustering, distillers, zap-list parsing) matches the oracle and
the reference.  No GPU work is issued here."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from peasoup_b200 import _lib


def test_library_exports_every_declared_symbol(psx):
    declared = _lib.declared_symbols()
    assert len(declared) >= 36
    missing = [s for s in declared if not hasattr(psx, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported
    # every declared function has a ctypes signature in the binding
    assert set(declared) == set(_lib.SIGNATURES)


def test_library_is_built_for_sm100a():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", _lib.LIB_PATH],
                         capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_status_and_version_strings(psx):
    assert b"sm_100a" in psx.psx_version()
    assert psx.psx_status_string(0) == b"ok"
    assert psx.psx_status_string(_lib.PSX_ERR_OVERFLOW) == b"output buffer too small"


def test_invalid_arguments_fail_loudly(psx):
    assert psx.psx_resampleII(None, None, 0, 1.0, 1e-4, None) == _lib.PSX_ERR_INVALID
    assert b"resample" in psx.psx_last_error()
    assert psx.psx_harmonic_sum(C.c_void_p(8), None, 16, 6, None) == _lib.PSX_ERR_INVALID
    cfg = _lib.SearchConfig()
    psx.psx_search_config_defaults(C.byref(cfg), 1000, 64e-6)  # not 2^k or 3*2^k
    h = C.c_void_p()
    assert psx.psx_search_create(C.byref(cfg), C.byref(h)) == _lib.PSX_ERR_INVALID
    psx.psx_search_config_defaults(C.byref(cfg), 1 << 16, 64e-6)
    cfg.nharmonics = 6
    assert psx.psx_search_create(C.byref(cfg), C.byref(h)) == _lib.PSX_ERR_INVALID
    assert b"nharmonics" in psx.psx_last_error()
    # the library's own transform: batched, 2^19 .. 2^27 or 3 * 2^17 .. 3 * 2^23
    # points
    for n, mode in ((1 << 16, _lib.PSX_MODE_BATCHED), (3 << 16, _lib.PSX_MODE_BATCHED),
                    (3 << 24, _lib.PSX_MODE_BATCHED),
                    (1 << 28, _lib.PSX_MODE_BATCHED), (1 << 20, _lib.PSX_MODE_PLAIN)):
        psx.psx_search_config_defaults(C.byref(cfg), n, 64e-6)
        cfg.mode, cfg.fft_form = mode, 3
        assert psx.psx_search_create(C.byref(cfg), C.byref(h)) == _lib.PSX_ERR_INVALID
        assert b"fft_form 3" in psx.psx_last_error()
    # the resample inside cuFFT (LTO load callbacks) is refused, not emulated
    psx.psx_search_config_defaults(C.byref(cfg), 1 << 20, 64e-6)
    cfg.use_fft_callback = 1
    assert psx.psx_search_create(C.byref(cfg), C.byref(h)) == _lib.PSX_ERR_UNSUPPORTED
    assert b"use_fft_callback" in psx.psx_last_error()
    cfg.use_fft_callback = 0
    cfg.fft_form = 4
    assert psx.psx_search_create(C.byref(cfg), C.byref(h)) == _lib.PSX_ERR_INVALID
    cfg.fft_form = 0
    for g in (-1, 17):
        cfg.group_dms = g
        assert psx.psx_search_create(C.byref(cfg), C.byref(h)) == _lib.PSX_ERR_INVALID
        assert b"group_dms" in psx.psx_last_error()
    cfg.group_dms = 0
    assert psx.psx_search_set_priority(None, 1) == _lib.PSX_ERR_INVALID


def test_no_cpu_fallback_without_device(psx):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    cfg = _lib.SearchConfig()
    psx.psx_search_config_defaults(C.byref(cfg), 1 << 16, 64e-6)
    h = C.c_void_p()
    rc = psx.psx_search_create(C.byref(cfg), C.byref(h))
    assert rc in (_lib.PSX_ERR_CUDA, _lib.PSX_ERR_ALLOC)
    from peasoup_b200 import transforms
    with pytest.raises(_lib.PsxError):
        transforms.DeviceTimeSeries(16)


def test_footprint_model(psx):
    from peasoup_b200.search import SearchParams, footprint
    small = footprint(SearchParams(fft_size=1 << 20, tsamp=64e-6))
    big = footprint(SearchParams(fft_size=1 << 23, tsamp=76e-6))
    assert 0 < small < big
    plain = footprint(SearchParams(fft_size=1 << 23, tsamp=76e-6, mode="plain"))
    assert plain < big
    # grouped prologues (default 4 rows up to 2^22 points) hold two sets of
    # rows; longer transforms do not group unless asked
    N = 1 << 22
    grouped = footprint(SearchParams(fft_size=N, tsamp=64e-6, batch=16))
    single = footprint(SearchParams(fft_size=N, tsamp=64e-6, batch=16, group_dms=1))
    assert single + 2 * 4 * 12 * N < grouped < single + 2 * 4 * 24 * N
    assert footprint(SearchParams(fft_size=N, tsamp=64e-6, batch=16, group_dms=8)) > grouped
    big1 = footprint(SearchParams(fft_size=1 << 23, tsamp=64e-6, batch=16))
    assert big1 == footprint(SearchParams(fft_size=1 << 23, tsamp=64e-6, batch=16, group_dms=1))
    assert big1 < footprint(SearchParams(fft_size=1 << 23, tsamp=64e-6, batch=16, group_dms=4))


def test_zaplist_parsing(psx):
    fd, path = tempfile.mkstemp(suffix=".txt")
    with os.fdopen(fd, "w") as f:
        f.write("50.000 0.100\n\n100.00 0.15\n  150.00   0.15  extra\n")
    try:
        n = C.c_size_t()
        assert psx.psx_read_zaplist(path.encode(), None, None, 0, C.byref(n)) == 0
        assert n.value == 3
        fr = np.zeros(3, np.float32)
        wd = np.zeros(3, np.float32)
        assert psx.psx_read_zaplist(path.encode(), fr.ctypes.data, wd.ctypes.data, 3,
                                    C.byref(n)) == 0
        assert list(fr) == [50.0, 100.0, 150.0]
        assert np.allclose(wd, [0.1, 0.15, 0.15])
        assert psx.psx_read_zaplist(path.encode(), fr.ctypes.data, wd.ctypes.data, 2,
                                    C.byref(n)) == _lib.PSX_ERR_OVERFLOW
    finally:
        os.unlink(path)
    assert psx.psx_read_zaplist(b"/nonexistent/zaplist", None, None, 0,
                                C.byref(C.c_size_t())) == _lib.PSX_ERR_IO


def test_server_needs_a_device(psx):
    """Without a CUDA device the server refuses to start (no CPU fallback)."""
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from peasoup_b200._lib import PSX_ERR_CUDA, ServerConfig
    cfg = ServerConfig(device=0, hbm_budget=1 << 30, max_active=2, max_queue=8)
    h = C.c_void_p()
    assert psx.psx_server_create(C.byref(cfg), C.byref(h)) == PSX_ERR_CUDA
    bad = ServerConfig(device=0, hbm_budget=0, max_active=0, max_queue=0)
    assert psx.psx_server_create(C.byref(bad), C.byref(h)) == 1
    bad_policy = ServerConfig(device=0, hbm_budget=1 << 30, max_active=2, max_queue=8, policy=3)
    assert psx.psx_server_create(C.byref(bad_policy), C.byref(h)) == 1
    assert b"policy" in psx.psx_last_error()


def test_binding_constants_match_header():
    import re
    hdr = open(os.path.join(os.path.dirname(_lib.LIB_PATH), "..", "include",
                            "peasoup_b200.h")).read()
    assert int(re.search(r"#define PSX_HARM_SHAPES (\d+)", hdr).group(1)) == _lib.PSX_HARM_SHAPES


def test_two_pass_transform_lengths(psx):
    """Host rule of the two-pass transform (fft_form 3): batched mode,
    2^19 .. 2^27 or 3 * 2^17 .. 3 * 2^23 points; a configuration outside it
    has no footprint (it is rejected before any device work)."""
    cfg = _lib.SearchConfig()
    ok = [1 << 19, 1 << 23, 1 << 25, 1 << 26, 1 << 27, 3 << 17, 3 << 20, 3 << 23]
    bad = [1 << 18, 1 << 28, 3 << 16, 3 << 24, 5 << 20, 1000]
    for n in ok + bad:
        psx.psx_search_config_defaults(C.byref(cfg), n, 64e-6)
        cfg.mode, cfg.fft_form = _lib.PSX_MODE_BATCHED, 3
        fp = psx.psx_search_footprint(C.byref(cfg))
        assert (fp > 0) == (n in ok), (n, fp)
    # the default form picks it where it applies, and the footprint then has
    # no batched cuFFT work areas
    psx.psx_search_config_defaults(C.byref(cfg), 1 << 23, 64e-6)
    cfg.mode, cfg.batch = _lib.PSX_MODE_BATCHED, 32
    cfg.fft_form = 0
    own = psx.psx_search_footprint(C.byref(cfg))
    cfg.fft_form = 1
    lib = psx.psx_search_footprint(C.byref(cfg))
    assert 0 < own < lib
