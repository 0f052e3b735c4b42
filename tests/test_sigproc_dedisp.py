"""Producer side on the CPU: the SIGPROC reader and DM-list reader of the
C ABI against the reference's own reader (oracle/_ref) and an independent
parse; the dedispersion plan's host arithmetic (delay table, DM list, max
delay) against the oracle, bit for bit; the oracle's dedispersion against
known answers (planted dispersed impulses, the tutorial filterbank's
pulsar at DM 30)."""
import ctypes as C
import os

import numpy as np
import pytest

from peasoup_b200 import _lib, sigproc

# The reference's example filterbank (250 ms pulsar at DM 30), as the
# oracle's build stages it beside the reference's built libraries.
TUTORIAL = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                        "_ref", "tutorial.fil")


def _hdr_dict(h):
    out = {f: getattr(h, f) for f, _ in _lib.SigprocHeader._fields_}
    out["source_name"] = h.source_name.decode()
    out["rawdatafile"] = h.rawdatafile.decode()
    return out


@pytest.fixture(scope="module")
def fil_file(tmp_path_factory, psx):
    """An 8-bit file with every header keyword set."""
    path = str(tmp_path_factory.mktemp("fil") / "all_keys.fil")
    rng = np.random.default_rng(5)
    rows = rng.integers(0, 256, (1000, 32), dtype=np.uint8)
    sigproc.write_filterbank(path, rows, source_name="J0000+0000", rawdatafile="raw.dat",
                             az_start=12.5, za_start=33.25, src_raj=123456.78,
                             src_dej=-123456.5, tstart=60000.123456789, tsamp=64e-6,
                             period=0.0123, fch1=1400.0, foff=-0.5, refdm=17.5, nchans=32,
                             telescope_id=6, machine_id=10, data_type=1, ibeam=3, nbeams=13,
                             nbits=8, barycentric=1, pulsarcentric=0, nbins=0, nifs=1,
                             npuls=0, signed_data=1)
    return path, rows


def test_header_round_trip_and_independent_parse(fil_file, oracle):
    path, rows = fil_file
    h = _hdr_dict(sigproc.read_header(path))
    ind = oracle.parse_sigproc_header(path)
    for k, v in ind.items():
        assert h[k] == v, k
    assert h["nsamples"] == rows.shape[0]            # from the file size
    assert h["header_size"] + rows.size == os.path.getsize(path)
    assert h["source_name"] == "J0000+0000" and h["signed_data"] == 1


def test_header_matches_reference_reader(fil_file, ref_host):
    path, _ = fil_file
    for p in [path] + ([TUTORIAL] if os.path.exists(TUTORIAL) else []):
        h = _hdr_dict(sigproc.read_header(p))
        ref = ref_host.ref_sigproc_header(p)
        for k, v in ref.items():
            assert h[k] == v, (p, k, h[k], v)


def test_reader_matches_reference_load_gulp(fil_file, ref_host):
    path, rows = fil_file
    cases = [(0, 0, 0, 1000), (100, 500, 150, 200), (0, 0, 900, 300), (10, 5000, 990, 50)]
    for seg_start, seg_n, start, n in cases:
        got, meta = ref_host.ref_filterbank_gulp(path, seg_start, seg_n, start, n, 32)
        fb = sigproc.SigprocFilterbank(path, seg_start, seg_n)
        k = fb.load_gulp(start, n)
        assert k * 32 == got.size and np.array_equal(fb.get_data(), got)
        assert np.array_equal(fb.get_data().reshape(-1, 32), rows[start:start + k])
        fb.size = 1 << 16
        mine = [fb.get_tsamp(), fb.get_fch1(), fb.get_foff(), fb.get_cfreq(),
                fb.get_start_sample(), fb.get_end_sample(), fb.get_effective_nsamps(),
                fb.get_total_nsamps(), fb.get_segment_pepoch()]
        assert mine == meta.tolist(), (seg_start, seg_n)


def test_start_past_end_raises(fil_file):
    with pytest.raises(_lib.PsxError):
        sigproc.SigprocFilterbank(fil_file[0], 5000, 10)


def test_bad_files(tmp_path, psx):
    p = tmp_path / "bad.fil"
    p.write_bytes(b"\x05\x00\x00\x00HELLO")
    with pytest.raises(_lib.PsxError):
        sigproc.read_header(str(p))
    with pytest.raises(_lib.PsxError):
        sigproc.read_header(str(tmp_path / "missing.fil"))
    # truncated before HEADER_END
    good = tmp_path / "t.fil"
    sigproc.write_header(str(good), sigproc.make_header(nchans=4, nbits=8, tsamp=1e-3,
                                                        fch1=100.0, foff=-1.0))
    data = good.read_bytes()
    (tmp_path / "trunc.fil").write_bytes(data[:-8])
    with pytest.raises(_lib.PsxError):
        sigproc.read_header(str(tmp_path / "trunc.fil"))


def test_dm_file_empty_lines_repeat(tmp_path, psx):
    p = tmp_path / "dms.txt"
    p.write_text("24.5\n25.0\n\n100.0\n")
    assert sigproc.read_dm_file(str(p)).tolist() == [24.5, 25.0, 25.0, 100.0]
    p.write_text("\n3.5\n")
    assert sigproc.read_dm_file(str(p)).tolist() == [0.0, 3.5]


def test_pack_matches_oracle_unpack(oracle):
    rng = np.random.default_rng(1)
    for nbits in (1, 2, 4, 8, 16):
        v = rng.integers(0, 1 << nbits, (37, 64), dtype=np.uint32)
        rows = sigproc.pack_samples(v, nbits)
        assert rows.shape == (37, 64 * nbits // 8)
        assert np.array_equal(oracle.unpack_rows(rows, 64, nbits), v)
        # the C restatement reads the same channel values
        for c in (0, 1, 5, 63):
            assert oracle._dedisp_lib().orc_sigproc_value(rows[3].ctypes.data, c, nbits) == v[3, c]


# -------------------------------------------------------- plan host arithmetic
PLAN_CASES = [(64, 320e-6, 1510.0, -1.09), (64, 64e-6, 1510.0, -1.09),
              (4096, 64e-6, 1500.0, -0.0732421875), (1024, 54.613e-6, 856.0 + 856.0, -0.8359375),
              (128, 256e-6, 400.0, -0.78125)]


def _plan(psx, nchans, tsamp, fch1, foff):
    h = C.c_void_p()
    assert psx.psx_dedisp_create(nchans, tsamp, fch1, foff, C.byref(h)) == 0
    return h


@pytest.mark.parametrize("case", PLAN_CASES)
def test_plan_delays_and_dm_list_equal_oracle(psx, oracle, case):
    nchans, tsamp, fch1, foff = case
    h = _plan(psx, *case)
    try:
        d = np.zeros(nchans, np.float32)
        assert psx.psx_dedisp_get_delay_table(h, d.ctypes.data) == 0
        assert np.array_equal(d, oracle.delay_table(nchans, tsamp, fch1, foff))
        assert d[0] == 0 and np.all(np.diff(d) > 0)
        for (lo, hi, w, tol) in ((0.0, 100.0, 64.0, 1.11), (2.0, 1000.0, 40.0, 1.25),
                                 (0.0, 0.0, 64.0, 1.11), (5.0, 5.5, 1000.0, 1.05)):
            assert psx.psx_dedisp_generate_dm_list(h, lo, hi, w, tol) == 0
            n = psx.psx_dedisp_get_dm_count(h)
            got = np.zeros(n, np.float32)
            assert psx.psx_dedisp_get_dm_list(h, got.ctypes.data, n) == 0
            want = oracle.dm_list(nchans, tsamp, fch1, foff, lo, hi, w, tol)
            assert np.array_equal(got, want)
            assert got[0] == np.float32(lo) and got[-1] >= np.float32(hi)
            assert n == 1 or (got[-2] < np.float32(hi) and np.all(np.diff(got) > 0))
            assert psx.psx_dedisp_get_max_delay(h) == oracle.max_delay(d, got)
    finally:
        psx.psx_dedisp_destroy(h)


def test_dm_step_meets_the_smearing_budget(oracle):
    """Each step solves the smearing equation it restates."""
    nchans, tsamp, fch1, foff, w, tol = 64, 64e-6, 1510.0, -1.09, 64.0, 1.11
    dms = oracle.dm_list(nchans, tsamp, fch1, foff, 0.0, 300.0, w, tol).astype(np.float64)
    ts = tsamp * 1e6
    f = (fch1 + (nchans // 2 - 0.5) * foff) * 1e-3
    a = 8.3 * foff / f ** 3
    b = a * nchans / 4
    for p, x in zip(dms[:-1], dms[1:]):
        lhs = ts ** 2 + w ** 2 + (a * x) ** 2 + (b * (x - p)) ** 2
        rhs = tol ** 2 * (ts ** 2 + w ** 2 + (a * p) ** 2)
        assert abs(lhs - rhs) <= 1e-5 * rhs


def test_plan_rejects_bad_arguments(psx):
    h = C.c_void_p()
    assert psx.psx_dedisp_create(64, 64e-6, 1510.0, 1.09, C.byref(h)) == _lib.PSX_ERR_INVALID
    assert psx.psx_dedisp_create(0, 64e-6, 1510.0, -1.09, C.byref(h)) == _lib.PSX_ERR_INVALID
    assert psx.psx_dedisp_create(64, 64e-6, 100.0, -2.0, C.byref(h)) == _lib.PSX_ERR_INVALID
    h = _plan(psx, 64, 64e-6, 1510.0, -1.09)
    try:
        bad = np.array([1.0, -2.0], np.float32)
        assert psx.psx_dedisp_set_dm_list(h, bad.ctypes.data, 2) == _lib.PSX_ERR_INVALID
        assert psx.psx_dedisp_generate_dm_list(h, 0.0, 10.0, 64.0, 1.0) == _lib.PSX_ERR_INVALID
        out = np.zeros(16, np.float32)
        # no DM list yet, then too few samples for the largest delay; 3-bit input
        assert psx.psx_dedisp_execute(h, 1000, None, 8, out.ctypes.data, 1000, 0, None) != 0
        dms = np.array([0.0, 1000.0], np.float32)
        assert psx.psx_dedisp_set_dm_list(h, dms.ctypes.data, 2) == 0
        md = psx.psx_dedisp_get_max_delay(h)
        assert psx.psx_dedisp_execute(h, md, C.c_void_p(16), 8, C.c_void_p(16), 1024, 0,
                                      None) == _lib.PSX_ERR_INVALID
        assert psx.psx_dedisp_execute(h, md + 100, C.c_void_p(16), 3, C.c_void_p(16), 1024, 0,
                                      None) == _lib.PSX_ERR_UNSUPPORTED
        # misaligned output pitch
        assert psx.psx_dedisp_execute(h, md + 100, C.c_void_p(16), 8, C.c_void_p(16), 102, 0,
                                      None) == _lib.PSX_ERR_INVALID
    finally:
        psx.psx_dedisp_destroy(h)


# ------------------------------------------------------------ oracle answers
@pytest.mark.parametrize("nbits", [1, 2, 4, 8, 16])
def test_oracle_recovers_planted_dispersed_impulses(oracle, nbits):
    """A unit impulse placed at t0 + D(d, c) in every channel sums to nchans
    at t0 for trial d; the other trials see it smeared."""
    nchans, tsamp, fch1, foff = 64, 64e-6, 1510.0, -1.09
    delays = oracle.delay_table(nchans, tsamp, fch1, foff)
    dms = np.array([0.0, 37.5, 80.0, 150.0], np.float32)
    md = oracle.max_delay(delays, dms)
    ns = md + 400
    for d, dm in enumerate(dms):
        v = np.zeros((ns, nchans), np.uint32)
        t0 = 123
        for c in range(nchans):
            v[t0 + int(np.rint(np.float32(dm) * delays[c])), c] = 1
        out = oracle.dedisperse(sigproc.pack_samples(v, nbits), nbits, nchans, delays, dms,
                                raw=True)
        assert out.shape == (4, ns - md)
        assert out[d, t0] == nchans and out[d].sum() == nchans
        for e in range(4):
            if e != d:
                assert out[e].max() < nchans
        mapped = oracle.dedisperse(sigproc.pack_samples(v, nbits), nbits, nchans, delays, dms)
        m = (1 << nbits) - 1
        want = (np.float32(nchans) - np.float32(0.5 * nchans * m)) * \
            np.float32(1.0 / (m * np.sqrt(nchans))) + np.float32(0.5)
        assert mapped[d, t0] == want
        # a killed channel drops out of the sum
        km = np.ones(nchans, np.int32)
        km[[0, 17, 63]] = 0
        killed = oracle.dedisperse(sigproc.pack_samples(v, nbits), nbits, nchans, delays, dms,
                                   killmask=km, raw=True)
        assert killed[d, t0] == nchans - 3


@pytest.mark.skipif(not os.path.exists(TUTORIAL), reason="reference example data absent")
def test_oracle_on_tutorial_filterbank(oracle):
    """The reference's example filterbank holds a 250 ms pulsar at DM 30:
    the per-channel arrival times of the folded pulse, unpacked and delayed
    by the oracle's rules, fit DM 30 +- 1.5, and the dedispersed series
    carries the 4 Hz line and its harmonics."""
    h = oracle.parse_sigproc_header(TUTORIAL)
    assert (h["nbits"], h["nchans"], h["nsamples"]) == (2, 64, 187520)
    rows = np.fromfile(TUTORIAL, np.uint8, offset=h["header_size"]).reshape(-1, 16)
    un = oracle.unpack_rows(rows, 64, 2).astype(np.float64)
    ts = h["tsamp"]
    nb = 500
    b = ((np.arange(un.shape[0]) * ts / 0.25) % 1.0 * nb).astype(int)
    cnt = np.bincount(b, None, nb)
    profs = np.array([np.bincount(b, un[:, c], nb) / cnt for c in range(64)])
    ref = profs.mean(0) - profs.mean()
    shifts = []
    for pr in profs:
        cc = np.fft.irfft(np.fft.rfft(pr - pr.mean()) * np.conj(np.fft.rfft(ref)), nb)
        k = int(np.argmax(cc))
        y0, y1, y2 = cc[(k - 1) % nb], cc[k], cc[(k + 1) % nb]
        s = k + 0.5 * (y0 - y2) / (y0 - 2 * y1 + y2)
        shifts.append((s - nb if s > nb / 2 else s) * 0.25 / nb)
    delays = oracle.delay_table(64, np.float32(ts), h["fch1"], h["foff"]).astype(np.float64)
    slope = np.polyfit(delays * ts, np.array(shifts), 1)[0]
    assert abs(slope - 30.0) < 1.5
    out = oracle.dedisperse(rows, 2, 64, oracle.delay_table(64, np.float32(ts), h["fch1"],
                                                            h["foff"]),
                            np.array([30.0], np.float32))[0]
    X = np.abs(np.fft.rfft(out - out.mean())) ** 2
    f = np.fft.rfftfreq(out.size, ts)
    X /= np.median(X)
    for k in (1, 2, 3):
        i = np.argmin(abs(f - 4.0 * k))
        assert X[i - 2:i + 3].max() > 100


def test_parse_header_from_memory(fil_file, psx):
    """psx_sigproc_parse_header on the file's leading bytes gives the
    header read_header gives (bar nsamples, which needs the file size);
    too few bytes ask for more; foreign bytes are rejected."""
    path, _ = fil_file
    data = open(path, "rb").read()
    whole = sigproc.read_header(path)
    h = _lib.SigprocHeader()
    assert psx.psx_sigproc_parse_header(data, len(data), C.byref(h)) == 0
    a, b = _hdr_dict(h), _hdr_dict(whole)
    a.pop("nsamples"), b.pop("nsamples")
    assert a == b
    assert psx.psx_sigproc_parse_header(data, 40, C.byref(h)) == _lib.PSX_ERR_OVERFLOW
    assert psx.psx_sigproc_parse_header(b"\x03\x00\x00\x00abc" + bytes(200), 207,
                                        C.byref(h)) == _lib.PSX_ERR_IO


def test_timeseries_dump_equals_reference_writer(tmp_path, psx):
    """sigproc.write_timeseries writes the .dat and .inf files the
    reference's DispersionTrials::write_timeseries_to_file writes (an odd
    sample count drops its last sample; coordinates with unpadded seconds;
    fixed-point fields as the reference's stream leaves them)."""
    from oracle import oracle as O
    if not os.path.exists(O.REF_GPU_PATH):
        pytest.skip("reference library not built")
    rng = np.random.default_rng(9)
    block = rng.standard_normal((3, 1001)).astype(np.float32)
    dms = np.array([0.0, 12.5, 123.456], np.float32)
    cases = [(123405.5, -453012.25, 6, 10, 64, -1.09), (2830.0, 51200.75, 0, 0, 4096, -0.0732),
             (-10203.25, -5.5, 1, 2, 96, 1.5)]
    for n, (raj, dej, tel, mach, nch, foff) in enumerate(cases):
        hd = np.array([raj, dej, 60000.123456789, 6.4e-05, 1510.0, foff])
        hi = np.array([tel, mach, nch], np.int32)
        for idx in range(3):
            ref_dir, our_dir = tmp_path / f"ref{n}{idx}", tmp_path / f"our{n}{idx}"
            ref_dir.mkdir()
            our_dir.mkdir()
            assert O.ref_write_timeseries(str(ref_dir), "stem", block, dms, idx, hd, hi,
                                          "J0000+0000") == 0
            h = sigproc.make_header(src_raj=raj, src_dej=dej, tstart=60000.123456789,
                                    tsamp=6.4e-05, fch1=1510.0, foff=foff, telescope_id=tel,
                                    machine_id=mach, nchans=nch, source_name="J0000+0000")
            sigproc.write_timeseries(str(our_dir), "stem", block[idx], dms[idx], h)
            names = sorted(os.listdir(ref_dir))
            assert names == sorted(os.listdir(our_dir)) and len(names) == 2
            for fn in names:
                a = open(ref_dir / fn, "rb").read()
                b = open(our_dir / fn, "rb").read()
                if fn.endswith(".inf"):
                    a = a.replace(str(ref_dir).encode(), b"DIR")
                    b = b.replace(str(our_dir).encode(), b"DIR")
                assert a == b, fn
