"""Dedispersion on the GPU against the oracle, bit for bit: every input
width (1, 2, 4, 8, 16 bits), raw and mapped output, sorted, generated and
unsorted DM lists (the wide-spread window path), killed channels, more
channels than a packed 16-bit accumulator holds (4096 at 8 bits, 4400 at
4 bits, where bytes are first summed as they stand), DM counts that do
not fill a CTA, a single output sample, host and device input; then the
Dedisperser class on a file, and the whole program (run) on a synthetic
tutorial-shaped filterbank and on the reference's own example filterbank:
the pulsars are found, and the candidates equal a search of the oracle's
dedispersed block."""
import ctypes as C
import os

import numpy as np
import pytest

from peasoup_b200 import _lib, sigproc, synth

pytestmark = pytest.mark.gpu


def _plan(psx, nchans, tsamp, fch1, foff):
    h = C.c_void_p()
    assert psx.psx_dedisp_create(nchans, tsamp, fch1, foff, C.byref(h)) == 0
    return h


def _run(psx, torch, h, rows, nbits, ndm, nout, raw, host=False):
    pitch = (nout + 3) // 4 * 4 + 4
    out = torch.full((ndm, pitch), -7.0, dtype=torch.float32, device="cuda")
    flags = _lib.PSX_DEDISP_RAW if raw else 0
    if host:
        rc = psx.psx_dedisp_execute_host(h, rows.shape[0], rows.ctypes.data, nbits,
                                         C.c_void_p(out.data_ptr()), pitch, flags, None)
    else:
        d_rows = torch.from_numpy(rows).cuda()
        rc = psx.psx_dedisp_execute(h, rows.shape[0], C.c_void_p(d_rows.data_ptr()), nbits,
                                    C.c_void_p(out.data_ptr()), pitch, flags, None)
    assert rc == 0, psx.psx_last_error()
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    assert np.all(o[:, nout:] == -7.0)  # nothing past the series is written
    return o[:, :nout]


CASES = [
    # nchans, nbits, tsamp, fch1, foff, dm list, nsamps past max delay
    (64, 2, 320e-6, 1510.0, -1.09, "gen:0:120", 3000),
    (64, 8, 64e-6, 1510.0, -1.09, "gen:0:300", 5000),
    (96, 4, 64e-6, 1400.0, -1.5, "gen:10:200", 2049),
    (64, 1, 64e-6, 1510.0, -1.09, "sorted:13", 1111),
    (32, 16, 128e-6, 1200.0, -2.0, "sorted:9", 1500),
    (64, 8, 64e-6, 1510.0, -1.09, "unsorted:2000:21", 700),
    (4096, 8, 64e-6, 1500.0, -0.0732421875, "sorted:8", 777),
    (300, 8, 64e-6, 1500.0, -0.5, "sorted:3", 1),
    (4400, 4, 64e-6, 1500.0, -300.0 / 4400, "sorted:3", 300),
    (64, 8, 64e-6, 1510.0, -1.09, "zero", 513),
]


def _dm_list(psx, h, spec, oracle, case):
    nchans, nbits, tsamp, fch1, foff = case[:5]
    rng = np.random.default_rng(len(spec))
    if spec.startswith("gen:"):
        _, lo, hi = spec.split(":")
        assert psx.psx_dedisp_generate_dm_list(h, float(lo), float(hi), 64.0, 1.11) == 0
        n = psx.psx_dedisp_get_dm_count(h)
        dms = np.zeros(n, np.float32)
        psx.psx_dedisp_get_dm_list(h, dms.ctypes.data, n)
        assert np.array_equal(dms, oracle.dm_list(nchans, tsamp, fch1, foff, float(lo),
                                                  float(hi), 64.0, 1.11))
        return dms
    if spec.startswith("sorted:"):
        dms = np.sort(rng.uniform(0, 120, int(spec.split(":")[1]))).astype(np.float32)
    elif spec.startswith("unsorted:"):
        _, hi, n = spec.split(":")
        dms = rng.uniform(0, float(hi), int(n)).astype(np.float32)
    else:
        dms = np.zeros(1, np.float32)
    assert psx.psx_dedisp_set_dm_list(h, dms.ctypes.data, dms.size) == 0
    return dms


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}ch-{c[1]}bit-{c[5]}" for c in CASES])
def test_dedisperse_equals_oracle(psx, cuda, oracle, case):
    torch = cuda
    nchans, nbits, tsamp, fch1, foff, spec, extra = case
    h = _plan(psx, nchans, tsamp, fch1, foff)
    try:
        dms = _dm_list(psx, h, spec, oracle, case)
        delays = oracle.delay_table(nchans, tsamp, fch1, foff)
        md = psx.psx_dedisp_get_max_delay(h)
        assert md == oracle.max_delay(delays, dms)
        ns = md + extra
        rng = np.random.default_rng(nchans + nbits)
        v = rng.integers(0, 1 << nbits, (ns, nchans), dtype=np.uint32)
        rows = sigproc.pack_samples(v, nbits)
        want_raw = oracle.dedisperse(rows, nbits, nchans, delays, dms, raw=True)
        want = oracle.dedisperse(rows, nbits, nchans, delays, dms)
        got_raw = _run(psx, torch, h, rows, nbits, dms.size, extra, True)
        assert np.array_equal(got_raw, want_raw)
        got = _run(psx, torch, h, rows, nbits, dms.size, extra, False, host=True)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        # killed channels
        km = (rng.random(nchans) > 0.2).astype(np.int32)
        assert psx.psx_dedisp_set_killmask(h, km.ctypes.data) == 0
        got = _run(psx, torch, h, rows, nbits, dms.size, extra, True)
        assert np.array_equal(got, oracle.dedisperse(rows, nbits, nchans, delays, dms,
                                                     killmask=km, raw=True))
        zero = np.zeros(nchans, np.int32)
        assert psx.psx_dedisp_set_killmask(h, zero.ctypes.data) == 0
        assert np.all(_run(psx, torch, h, rows, nbits, dms.size, extra, True) == 0)
        assert psx.psx_dedisp_set_killmask(h, None) == 0
        assert np.array_equal(_run(psx, torch, h, rows, nbits, dms.size, extra, True), want_raw)
    finally:
        psx.psx_dedisp_destroy(h)


def test_dedisperser_class_on_a_file(psx, cuda, oracle, tmp_path):
    from peasoup_b200.dedisperse import Dedisperser
    spec = synth.FilterbankSpec(nsamps=20000, tsamp=64e-6, nbits=4, dm=50.0,
                                pulsars=[synth.Pulsar(0.0371, 0.0, 0.03, 2.0)])
    v = synth.filterbank_values(spec, seed=3)
    path = str(tmp_path / "f.fil")
    sigproc.write_filterbank(path, sigproc.pack_samples(v, 4), nchans=64, nbits=4,
                             tsamp=64e-6, fch1=synth.FCH1_MHZ, foff=synth.FOFF_MHZ, tstart=60000.0,
                             nifs=1, data_type=1)
    fb = sigproc.SigprocFilterbank(path, 1000, 15000)
    dd = Dedisperser(fb)
    dd.generate_dm_list(0.0, 100.0, 64.0, 1.11)
    dms = dd.get_dm_list()
    tr = dd.dedisperse(gulp=4096)
    rows = sigproc.pack_samples(v[1000:16000], 4)
    want = oracle.dedisperse(rows, 4, 64, dd.get_delay_table(), dms)
    assert tr.get_nsamps() == 15000 - dd.get_max_delay()
    assert np.array_equal(tr.to_host().view(np.uint32), want.view(np.uint32))
    # the trial nearest DM 50 carries the most pulse power
    power = [np.abs(np.fft.rfft(r - r.mean()))[1:].max() for r in want]
    assert abs(dms[int(np.argmax(power))] - 50.0) < 12.0
    dd.close()


def _family(f, f0):
    """f is a harmonic (up to 16) or sub-harmonic of f0, within 1e-3."""
    r = f / f0 if f >= f0 else f0 / f
    return round(r) <= 16 and abs(r - round(r)) < 1e-3 * r


def test_whole_program_on_synthetic_tutorial(psx, cuda, oracle, tmp_path):
    """Tutorial shape (2-bit, 64 channels, 320 us) with the tutorial's
    250 ms pulsar and a 4.7 ms pulsar, both at DM 30.  run()'s outputs equal
    search_to_outputs on the oracle's dedispersion of the same file; the
    250 ms pulsar is found; the 4.7 ms pulsar, whose harmonics a few DM steps
    of smearing wash out, peaks within 7 of DM 30.  (A 250 ms pulse barely
    changes with DM in a 16-harmonic search, so its own best DM is not a
    known answer.)"""
    from peasoup_b200 import output, pipeline
    from peasoup_b200.search import SearchParams
    spec = synth.FilterbankSpec(nsamps=140000, tsamp=320e-6, nbits=2, dm=30.0,
                                pulsars=[synth.Pulsar(0.25, 0.0, 0.01, 0.9),
                                         synth.Pulsar(0.0047, 0.0, 0.1, 0.35)])
    v = synth.filterbank_values(spec, seed=11)
    path = str(tmp_path / "tut.fil")
    sigproc.write_filterbank(path, sigproc.pack_samples(v, 2), source_name="P: 250 ms, DM: 30",
                             nchans=64, nbits=2, tsamp=320e-6, fch1=1510.0, foff=-1.09,
                             tstart=50000.0, nifs=1, data_type=1)
    opts = pipeline.Options(path, outdir=str(tmp_path / "out"), dm_start=0.0, dm_end=60.0,
                            min_snr=8.0)
    nodes, sizes, scores, offsets, timers = pipeline.run(opts)
    xml = open(os.path.join(opts.outdir, "overview.xml")).read()
    for sec in ("header_parameters", "search_parameters", "segment_parameters", "dedispersion_trials",
                "candidates"):
        assert f"<{sec}" in xml
    assert os.path.getsize(os.path.join(opts.outdir, "candidates.peasoup")) > 0
    # the same search on the oracle's dedispersion of the file
    fb = sigproc.SigprocFilterbank(path)
    dms = oracle.dm_list(64, np.float32(320e-6), 1510.0, -1.09, 0.0, 60.0, 64.0, 1.11)
    delays = oracle.delay_table(64, np.float32(320e-6), 1510.0, -1.09)
    block = oracle.dedisperse(sigproc.pack_samples(v, 2), 2, 64, delays, dms)
    size = sigproc.prev_power_of_two(fb.get_effective_nsamps())
    cf = fb.get_cfreq()
    params = SearchParams(fft_size=size, tsamp=float(np.float32(320e-6)),
                          cfreq_hz=float(np.float32(float(np.float32(cf)) * 1e6)),
                          ch_bw_hz=float(np.float32(float(np.float32(-1.09)) * 1e6)),
                          min_snr=8.0, acc_pulse_width=float(np.float32(64.0 * 1e-6)))
    n2, s2, _, _, _ = pipeline.search_to_outputs(
        block, dms, params, str(tmp_path / "out2"), foff_mhz=float(np.float32(-1.09)),
        nchans=64, cfreq_mhz=cf, dm_chunk=len(dms))
    assert np.array_equal(nodes, n2) and np.array_equal(sizes, s2)
    # known answers
    top = nodes[output.roots(sizes)]
    assert any(_family(float(c["freq"]), 4.0) for c in top)
    fast = [c for c in top if _family(float(c["freq"]), 1.0 / 0.0047)]
    assert fast
    best = max(fast, key=lambda c: c["snr"])
    assert abs(best["dm"] - 30.0) <= 7.0, (best["dm"], best["snr"], best["freq"])


TUTORIAL = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                        "_ref", "tutorial.fil")


@pytest.mark.skipif(not os.path.exists(TUTORIAL),
                    reason="the reference's example filterbank is staged by the oracle's build")
def test_whole_program_on_tutorial_filterbank(psx, cuda, oracle, tmp_path):
    """The reference's example data (example_data/tutorial.fil: 2-bit, 64
    channels, 320 us, 187,520 samples, source "P: 250 ms, DM: 30") through
    the whole program as the reference's main runs it (header, segment,
    DM list 0..60, dedispersion into device memory, search, distillers,
    outputs): the candidates equal a search of the oracle's dedispersion of
    the same file, and the 4 Hz family is among the top candidates, its
    strongest detection at a DM trial near 30."""
    from peasoup_b200 import output, pipeline
    from peasoup_b200.search import SearchParams
    opts = pipeline.Options(TUTORIAL, outdir=str(tmp_path / "out"), dm_start=0.0, dm_end=60.0,
                            min_snr=8.0)
    nodes, sizes, scores, offsets, timers = pipeline.run(opts)
    assert os.path.getsize(os.path.join(opts.outdir, "candidates.peasoup")) > 0
    fb = sigproc.SigprocFilterbank(TUTORIAL)
    h = oracle.parse_sigproc_header(TUTORIAL)
    rows = np.fromfile(TUTORIAL, np.uint8, offset=h["header_size"]).reshape(-1, 16)
    ts = np.float32(h["tsamp"])
    dms = oracle.dm_list(64, ts, h["fch1"], h["foff"], 0.0, 60.0, 64.0, 1.11)
    delays = oracle.delay_table(64, ts, h["fch1"], h["foff"])
    block = oracle.dedisperse(rows, 2, 64, delays, dms)
    size = sigproc.prev_power_of_two(fb.get_effective_nsamps())
    cf = fb.get_cfreq()
    foff = float(np.float32(h["foff"]))
    params = SearchParams(fft_size=size, tsamp=float(ts),
                          cfreq_hz=float(np.float32(float(np.float32(cf)) * 1e6)),
                          ch_bw_hz=float(np.float32(foff * 1e6)),
                          min_snr=8.0, acc_pulse_width=float(np.float32(64.0 * 1e-6)))
    n2, s2, _, _, _ = pipeline.search_to_outputs(
        block, dms, params, str(tmp_path / "out2"), foff_mhz=foff, nchans=64, cfreq_mhz=cf,
        dm_chunk=len(dms))
    assert np.array_equal(nodes, n2) and np.array_equal(sizes, s2)
    top = nodes[output.roots(sizes)]
    fam = [c for c in top if _family(float(c["freq"]), 4.0)]
    print("tutorial: %d top candidates, 4 Hz family:" % len(top),
          [(float(c["dm"]), float(c["freq"]), float(c["snr"])) for c in fam[:8]])
    assert fam
    best = max(fam, key=lambda c: c["snr"])
    assert abs(best["dm"] - 30.0) <= 10.0, (best["dm"], best["snr"], best["freq"])


@pytest.mark.parametrize("nchans,nbits", [(64, 8), (4096, 8), (64, 2), (32, 16)])
def test_time_gulps_equal_one_pass(psx, cuda, oracle, nchans, nbits):
    """A scratch limit a few tiles long splits the series into time gulps
    (overlapping by the maximum delay); device and host input both stay bit
    for bit equal to the oracle."""
    torch = cuda
    tsamp, fch1, foff = 64e-6, 1500.0, -300.0 / nchans
    h = _plan(psx, nchans, tsamp, fch1, foff)
    try:
        dms = np.linspace(0.0, 40.0, 11).astype(np.float32)
        assert psx.psx_dedisp_set_dm_list(h, dms.ctypes.data, dms.size) == 0
        md = psx.psx_dedisp_get_max_delay(h)
        extra = 5000 + 333
        rng = np.random.default_rng(nchans)
        v = rng.integers(0, 1 << nbits, (md + extra, nchans), dtype=np.uint32)
        rows = sigproc.pack_samples(v, nbits)
        delays = oracle.delay_table(nchans, tsamp, fch1, foff)
        want = oracle.dedisperse(rows, nbits, nchans, delays, dms, raw=True)
        el = 2 if nbits == 16 else 1
        assert psx.psx_dedisp_set_scratch_limit(h, nchans * el * (md + 3000)) == 0
        assert np.array_equal(_run(psx, torch, h, rows, nbits, dms.size, extra, True), want)
        assert np.array_equal(_run(psx, torch, h, rows, nbits, dms.size, extra, True,
                                   host=True), want)
    finally:
        psx.psx_dedisp_destroy(h)


def test_cpp_dropin_headers(psx, cuda, oracle, tmp_path):
    """The drop-in C++ classes (SigprocFilterbank, read_header, Dedisperser,
    DispersionTrials), compiled with g++ as the reference's main program
    uses them: segment, generated DM list and killfile give the oracle's
    block bit for bit."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "dropin_dedisp")
    cmd = ["g++", "-O2", "-std=c++17", f"-I{root}/include", "-I/usr/local/cuda/include",
           f"{root}/tests/cpp/dropin_dedisp.cpp", f"-L{root}/peasoup_b200", "-lpeasoup_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{root}/peasoup_b200", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    spec = synth.FilterbankSpec(nsamps=30000, tsamp=128e-6, nbits=2, dm=20.0,
                                pulsars=[synth.Pulsar(0.0123, 0.0, 0.05, 1.0)])
    v = synth.filterbank_values(spec, seed=4)
    path = str(tmp_path / "d.fil")
    sigproc.write_filterbank(path, sigproc.pack_samples(v, 2), source_name="J1234+5678",
                             nchans=64, nbits=2, tsamp=128e-6, fch1=synth.FCH1_MHZ,
                             foff=synth.FOFF_MHZ, tstart=59000.5, nifs=1, data_type=1)
    kill = tmp_path / "kill.txt"
    km = np.ones(64, np.int32)
    km[[3, 40, 41]] = 0
    kill.write_text("\n".join(str(int(k)) for k in km) + "\n")
    out = str(tmp_path / "block.bin")
    r = subprocess.run([exe, path, "2000", "25000", "0", "50", out, "-", str(kill)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    ndm = int(np.frombuffer(raw, np.int32, 1, 0)[0])
    ns = int(np.frombuffer(raw, np.int64, 1, 4)[0])
    meta = np.frombuffer(raw, np.float32, 4, 28)
    dms = np.frombuffer(raw, np.float32, ndm, 44)
    block = np.frombuffer(raw, np.float32, ndm * ns, 44 + 4 * ndm).reshape(ndm, ns)
    fb = sigproc.SigprocFilterbank(path, 2000, 25000)
    assert list(meta) == [np.float32(fb.get_tsamp()), np.float32(fb.get_fch1()),
                          np.float32(fb.get_foff()), np.float32(fb.get_cfreq())]
    want_dms = oracle.dm_list(64, np.float32(128e-6), synth.FCH1_MHZ, synth.FOFF_MHZ, 0.0, 50.0,
                              64.0, 1.11)
    assert np.array_equal(dms, want_dms)
    delays = oracle.delay_table(64, np.float32(128e-6), synth.FCH1_MHZ, synth.FOFF_MHZ)
    want = oracle.dedisperse(sigproc.pack_samples(v[2000:27000], 2), 2, 64, delays, want_dms,
                             killmask=km)
    assert np.array_equal(block.view(np.uint32), want.view(np.uint32))


def test_whole_program_chunks_dm_file_killfile_zaplist(psx, cuda, tmp_path):
    """run() with a DM file (an empty line repeats the previous DM), a
    killfile and a zap list, once in one DM chunk and once in chunks of 4
    DM trials (the host-RAM rule): the candidates are the same apart from
    their DM indices, which restart in every chunk as the reference's do."""
    from peasoup_b200 import output, pipeline
    spec = synth.FilterbankSpec(nsamps=70000, tsamp=320e-6, nbits=2, dm=30.0,
                                pulsars=[synth.Pulsar(0.0047, 0.0, 0.1, 0.4)])
    v = synth.filterbank_values(spec, seed=12)
    path = str(tmp_path / "c.fil")
    sigproc.write_filterbank(path, sigproc.pack_samples(v, 2), nchans=64, nbits=2,
                             tsamp=320e-6, fch1=1510.0, foff=-1.09, tstart=50000.0, nifs=1,
                             data_type=1)
    dmf = tmp_path / "dms.txt"
    dmf.write_text("0\n10\n20\n\n28\n30\n32\n40\n50\n60\n")
    killf = tmp_path / "kill.txt"
    km = np.ones(64, np.int32)
    km[[5, 6, 60]] = 0
    killf.write_text("\n".join(str(int(k)) for k in km) + "\n")
    zapf = tmp_path / "zap.txt"
    zapf.write_text("50.0 0.5\n123.4 0.2\n")
    dms = sigproc.read_dm_file(str(dmf))
    assert dms.tolist() == [0, 10, 20, 20, 28, 30, 32, 40, 50, 60]
    res = {}
    for name, ram in (("one", 20.0), ("chunks", 4.5 * 70000 * 4 / 1e9)):
        opts = pipeline.Options(path, outdir=str(tmp_path / name), dm_file=str(dmf),
                                killfilename=str(killf), zapfilename=str(zapf), min_snr=7.0,
                                host_ram_limit_gb=ram)
        res[name] = pipeline.run(opts)
        assert "<dedispersion_trials" in open(tmp_path / name / "overview.xml").read()
    (n1, s1), (n2, s2) = res["one"][:2], res["chunks"][:2]
    assert np.array_equal(s1, s2) and len(n1) > 0
    for f in ("dm", "acc", "nh", "snr", "freq"):
        assert np.array_equal(n1[f], n2[f]), f
    # DM indices: positions in the whole list, then positions within chunks of 4
    pos = {float(d): i for i, d in reversed(list(enumerate(dms)))}
    assert all(int(c["dm_idx"]) < 4 for c in n2)
    assert all(int(c["dm_idx"]) == pos[float(c["dm"])] % 4 or float(c["dm"]) == 20.0
               for c in n2)
    top = n1[output.roots(s1)]
    best = max((c for c in top if _family(float(c["freq"]), 1.0 / 0.0047)),
               key=lambda c: c["snr"])
    assert abs(best["dm"] - 30.0) <= 2.0


def test_whole_program_timeseries_dump(psx, cuda, oracle, tmp_path):
    """run() with a dump directory writes every DM trial's series of every
    DM chunk (the oracle's dedispersion of that chunk, an even number of
    samples) and its .inf; with no_search nothing is searched and no output
    files appear."""
    from peasoup_b200 import pipeline
    v = synth.filterbank_values(synth.FilterbankSpec(nsamps=20001, tsamp=320e-6, nbits=2),
                                seed=13)
    path = str(tmp_path / "obs.fil")
    sigproc.write_filterbank(path, sigproc.pack_samples(v, 2), nchans=64, nbits=2, tsamp=320e-6,
                             fch1=1510.0, foff=-1.09, tstart=50000.0, nifs=1, data_type=1,
                             source_name="OBS")
    dmf = tmp_path / "dms.txt"
    dmf.write_text("0\n5.25\n30\n")
    dump = tmp_path / "dump"
    out = pipeline.run(pipeline.Options(path, outdir=str(tmp_path / "out"), dm_file=str(dmf),
                                        timeseries_dump_dir=str(dump), no_search=True,
                                        host_ram_limit_gb=2 * 20001 * 4 / 1e9 * 1.1))
    assert out is None and not (tmp_path / "out").exists()
    names = sorted(os.listdir(dump))
    assert names == ["obs_DM00000.000.dat", "obs_DM00000.000.inf", "obs_DM00005.250.dat",
                     "obs_DM00005.250.inf", "obs_DM00030.000.dat", "obs_DM00030.000.inf"]
    # chunks of two DM trials, each with its own maximum delay and length
    delays = oracle.delay_table(64, np.float32(320e-6), 1510.0, -1.09)
    # the header has no nsamples: the count comes from the file size as the
    # reference forms it (bytes / nchans * 8 / nbits), 20000 of the 20001
    total = sigproc.SigprocFilterbank(path).get_total_nsamps()
    assert total == 20000
    rows = sigproc.pack_samples(v[:total], 2)
    want = [oracle.dedisperse(rows, 2, 64, delays, np.array(c, np.float32))
            for c in ([0.0, 5.25], [30.0])]
    series = [want[0][0], want[0][1], want[1][0]]
    assert len(series[0]) != len(series[2])
    for i, dm in enumerate(("00000.000", "00005.250", "00030.000")):
        got = np.fromfile(dump / f"obs_DM{dm}.dat", np.float32)
        n = series[i].size - series[i].size % 2
        assert got.size == n and np.array_equal(got.view(np.uint32), series[i][:n].view(np.uint32))
        inf = open(dump / f"obs_DM{dm}.inf").read()
        assert f"Number of bins in the time series      =  {n}\n" in inf
        assert "Object being observed                  =  OBS\n" in inf
