"""GPU parity of every single stage: the product (through its C ABI, via the
transform-API mirror) against the FP64 oracle, and against the reference's
own CUDA build where oracle/_ref is present.

Tolerances (stated per stage):
  * resampled series: bit-exact (index arithmetic in FP64);
  * spectra (FFT, amplitude, interbin, median, dereddened, harmonic sums):
    within 1e-5 relative to the spectrum's RMS against FP64;
  * against the reference build: the same operations in the same order,
    so exact equality is required except where the reference reduces in
    a different order (statistics: 1e-6 relative).
"""
import os
import tempfile

import numpy as np
import pytest

from helpers import err_vs_rms, rel_err

pytestmark = pytest.mark.gpu

TS = np.float32(64e-6)
ACCS = [-500.0, -123.4, -12.0, 0.0, 12.0, 125.5, 500.0]


@pytest.fixture(scope="module")
def T(cuda, psx):
    from peasoup_b200 import transforms as T
    return T


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("n", [1 << 16, 3 << 15, (1 << 20) + 4])
@pytest.mark.parametrize("acc", ACCS)
def test_resampleII_bit_exact_vs_oracle(T, oracle, n, acc):
    x = np.arange(n, dtype=np.float32) if n <= (1 << 24) else None
    a = T.DeviceTimeSeries.from_host(x, float(TS))
    b = T.DeviceTimeSeries(n, float(TS))
    T.TimeDomainResampler().resampleII(a, b, n, acc)
    got = _host(b.data).astype(np.int64)
    want = oracle.resampleII_index(n, acc, float(TS), fused=1).astype(np.int64)
    assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} index mismatches"


@pytest.mark.parametrize("acc", ACCS)
def test_resample_centred_vs_oracle(T, oracle, acc):
    n = 1 << 18
    x = np.arange(n, dtype=np.float32)
    a = T.DeviceTimeSeries.from_host(x, float(TS))
    b = T.DeviceTimeSeries(n, float(TS))
    T.TimeDomainResampler().resample(a, b, n, acc)
    got = _host(b.data).astype(np.int64)
    v0 = oracle.resample_index(n, acc, float(TS), fused=0).astype(np.int64)
    v1 = oracle.resample_index(n, acc, float(TS), fused=1).astype(np.int64)
    # mathematically identical to resampleII; the rounding of the centred
    # form is compiler-dependent, so either contraction is accepted
    assert np.array_equal(got, v0) or np.array_equal(got, v1)


def test_resampleII_vs_reference(T, ref_gpu):
    for n in (1 << 18, 3 << 16):
        x = np.arange(n, dtype=np.float32)
        for acc in ACCS:
            want = ref_gpu.ref_resampleII(x, acc, float(TS))
            a = T.DeviceTimeSeries.from_host(x, float(TS))
            b = T.DeviceTimeSeries(n, float(TS))
            T.TimeDomainResampler().resampleII(a, b, n, acc)
            assert np.array_equal(_host(b.data), want), (n, acc)


def test_resample_centred_vs_reference(T, ref_gpu):
    n = 1 << 18
    x = np.arange(n, dtype=np.float32)
    for acc in ACCS:
        want = ref_gpu.ref_resample(x, acc, float(TS))
        a = T.DeviceTimeSeries.from_host(x, float(TS))
        b = T.DeviceTimeSeries(n, float(TS))
        T.TimeDomainResampler().resample(a, b, n, acc)
        assert np.array_equal(_host(b.data), want), acc


@pytest.mark.parametrize("n", [1 << 14, 3 << 13, 1 << 20])
def test_fft_r2c_c2r_vs_oracle(T, oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n).astype(np.float32)
    fft = T.CuFFTerR2C(n)
    fs = T.DeviceFourierSeries(n // 2 + 1, 1.0)
    fft.execute(_dev(x), fs.data)
    got = _host(fs.data).view(np.complex64)
    want = oracle.rfft(x.astype(np.float64))
    assert err_vs_rms(got, want) < 1e-5
    ifft = T.CuFFTerC2R(n)
    y = _dev(np.zeros(n, np.float32))
    ifft.execute(fs.data, y)
    back = _host(y)
    assert err_vs_rms(back, n * x.astype(np.float64)) < 1e-5


@pytest.mark.parametrize("n,batch", [(1 << 12, 3), (3 << 10, 1)])
def test_fft_c2c_both_directions(T, n, batch):
    """CuFFTerC2C (ffter.hpp:33-53): the forward transform against FP64
    numpy (within 1e-5 of the RMS), and forward then inverse gives n times
    the input (unnormalised, as cufftExecC2C)."""
    rng = np.random.default_rng(n + batch)
    z = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(
        np.complex64)
    fft = T.CuFFTerC2C(n, batch)
    assert fft.get_output_size() == n
    a, b = _dev(z.view(np.float32)), _dev(np.zeros((batch, 2 * n), np.float32))
    fft.execute(a, b, -1)
    got = _host(b).view(np.complex64)
    want = np.fft.fft(z.astype(np.complex128), axis=1)
    assert err_vs_rms(got, want) < 1e-5
    fft.execute(b, b, +1)   # in place
    assert err_vs_rms(_host(b).view(np.complex64), n * z.astype(np.complex128)) < 1e-5
    from peasoup_b200._lib import PsxError
    with pytest.raises(PsxError):
        fft.execute(a, b, 0)


def test_fft_vs_reference(T, ref_gpu):
    rng = np.random.default_rng(3)
    n = 1 << 16
    x = rng.standard_normal(n).astype(np.float32)
    fs = T.DeviceFourierSeries(n // 2 + 1, 1.0)
    T.CuFFTerR2C(n).execute(_dev(x), fs.data)
    got = _host(fs.data).view(np.complex64)
    want = ref_gpu.ref_fft_r2c(x)
    assert err_vs_rms(got, want) < 1e-6


@pytest.mark.parametrize("way", [0, 1])
def test_form_vs_oracle_and_reference(T, oracle, way, request):
    rng = np.random.default_rng(5 + way)
    nb = (1 << 16) + 1
    X = (rng.standard_normal(nb) + 1j * rng.standard_normal(nb)).astype(np.complex64)
    X[9] = 0
    fs = T.DeviceFourierSeries(nb, 1.0, data=_dev(X.view(np.float32)))
    ps = T.DevicePowerSpectrum(fs)
    (T.SpectrumFormer().form_interpolated if way else T.SpectrumFormer().form)(fs, ps)
    got = _host(ps.data)
    want = (oracle.form_interbin if way else oracle.form_power)(X.astype(np.complex128))
    assert rel_err(got, want) < 1e-5
    if os.path.exists(oracle.REF_GPU_PATH):
        ref = oracle.ref_form(X, bool(way))
        assert np.array_equal(got, ref), f"{np.count_nonzero(got != ref)} bins differ"


def _red_amp(rng, nb):
    return (np.abs(rng.standard_normal(nb) + 1j * rng.standard_normal(nb)) *
            (1 + 50.0 / (1 + np.arange(nb) / 40.0))).astype(np.float32)


@pytest.mark.parametrize("nb", [(1 << 16) + 1, (3 << 15) + 1, (1 << 20) + 1, (1 << 26) + 1])
def test_running_median_vs_oracle(T, oracle, nb):
    """The 5/25/125-bin running median against FP64; 2^26 + 1 bins is the
    spectrum of a 2^27-point segment (256 MB, twice the L2)."""
    rng = np.random.default_rng(nb)
    amp = _red_amp(rng, nb)
    bw = float(np.float32(1.0 / np.float32(np.float32(2 * (nb - 1)) * TS)))
    ps = T.DevicePowerSpectrum(nb, bw, data=_dev(amp))
    d = T.Dereddener(nb)
    d.calculate_median(ps)
    got = _host(d.median)
    want = oracle.running_median(amp.astype(np.float64), bw)
    assert rel_err(got, want) < 1e-5


def test_running_median_and_deredden_vs_reference(T, ref_gpu):
    rng = np.random.default_rng(21)
    for nb in ((1 << 16) + 1, (1 << 19) + 1):
        amp = _red_amp(rng, nb)
        bw = float(np.float32(1.0 / np.float32(np.float32(2 * (nb - 1)) * TS)))
        ps = T.DevicePowerSpectrum(nb, bw, data=_dev(amp))
        d = T.Dereddener(nb)
        d.calculate_median(ps)
        got = _host(d.median)
        want = ref_gpu.ref_running_median(amp, bw)
        assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} median bins differ"
        X = (rng.standard_normal(nb) + 1j * rng.standard_normal(nb)).astype(np.complex64)
        fs = T.DeviceFourierSeries(nb, bw, data=_dev(X.view(np.float32)))
        d.deredden(fs)
        gotX = _host(fs.data).view(np.complex64)
        wantX = ref_gpu.ref_deredden(X, amp, bw)
        assert np.array_equal(gotX, wantX)


def test_fused_deredden_matches_two_step(T, psx):
    import ctypes as C
    import torch
    rng = np.random.default_rng(4)
    nb = (1 << 18) + 1
    amp = _red_amp(rng, nb)
    bw = float(np.float32(1.0 / np.float32(np.float32(2 * (nb - 1)) * TS)))
    X = (rng.standard_normal(nb) + 1j * rng.standard_normal(nb)).astype(np.complex64)
    fs = T.DeviceFourierSeries(nb, bw, data=_dev(X.view(np.float32)))
    ps = T.DevicePowerSpectrum(nb, bw, data=_dev(amp))
    d = T.Dereddener(nb)
    d.calculate_median(ps)
    d.deredden(fs)
    two = _host(fs.data)
    Y = _dev(X.view(np.float32))
    scratch = torch.zeros(psx.psx_running_median_scratch_bytes(nb) // 4 + 1, device="cuda")
    rc = psx.psx_deredden(C.c_void_p(Y.data_ptr()), C.c_void_p(ps.data.data_ptr()), nb, bw,
                          0.05, 0.5, C.c_void_p(scratch.data_ptr()), None)
    assert rc == 0
    assert np.array_equal(_host(Y), two)


def test_zap_vs_oracle_and_reference(T, oracle):
    rng = np.random.default_rng(8)
    nb = (1 << 16) + 1
    bw = float(np.float32(1.0 / np.float32(np.float32(1 << 17) * TS)))
    X = (rng.standard_normal(nb) + 1j * rng.standard_normal(nb)).astype(np.complex64)
    zf = np.array([0.3, 17.25, 50.0, 100.0, 1990.0, 5000.0], np.float32)
    zw = np.array([0.05, 0.1, 0.1, 0.15, 20.0, 1.0], np.float32)
    fd, zp = tempfile.mkstemp(suffix=".txt")
    with os.fdopen(fd, "w") as f:
        for a, b in zip(zf, zw):
            f.write(f"{a:.3f} {b:.3f}\n")
    try:
        fs = T.DeviceFourierSeries(nb, bw, data=_dev(X.view(np.float32)))
        T.Zapper(zp).zap(fs)
        got = _host(fs.data).view(np.complex64)
        want = oracle.zap(X.astype(np.complex128), float(np.float32(bw)), zf, zw)
        assert np.array_equal(got.astype(np.complex128), want.astype(np.complex64).astype(np.complex128))
        if os.path.exists(oracle.REF_GPU_PATH):
            assert np.array_equal(got, oracle.ref_zap(X, bw, zp))
    finally:
        os.unlink(zp)


def test_stats_normalise_baseline(T, oracle):
    rng = np.random.default_rng(9)
    p = (np.abs(rng.standard_normal((1 << 20) + 1)) * 3 + 1).astype(np.float32)
    m, r, s = T.stats.stats(_dev(p), p.size)
    wm, wr, ws = oracle.stats(p.astype(np.float64))
    assert abs(m - wm) / wm < 1e-6 and abs(r - wr) / wr < 1e-6 and abs(s - ws) / ws < 1e-5
    t = _dev(p)
    T.stats.normalise(t, 1.25, 0.75, p.size)
    got = _host(t)
    want = ((p - np.float32(1.25)) / np.float32(0.75)).astype(np.float32)
    assert np.array_equal(got, want)
    tim = (128 + 20 * rng.standard_normal(1 << 20)).astype(np.float32)
    ts = T.DeviceTimeSeries.from_host(tim, float(TS))
    passes = ts.remove_baseline()
    got = _host(ts.data)
    assert passes >= 1 and abs(float(np.mean(got.astype(np.float64)))) < 5e-7 * tim.size
    want, _ = oracle.remove_baseline(tim.astype(np.float64))
    assert err_vs_rms(got, want) < 1e-6
    if os.path.exists(oracle.REF_GPU_PATH):
        rm, rr, rs = oracle.ref_stats(p)
        assert abs(m - rm) / rm < 1e-6 and abs(r - rr) / rr < 1e-6
        t2 = _dev(p)
        T.stats.normalise(t2, 1.25, 0.75, p.size)
        assert np.array_equal(_host(t2), oracle.ref_normalise(p, 1.25, 0.75))


@pytest.mark.parametrize("nfolds", [1, 2, 3, 4, 5])
def test_harmonic_sums_vs_oracle(T, oracle, nfolds):
    rng = np.random.default_rng(nfolds)
    nb = (1 << 18) + 1
    s = rng.standard_normal(nb).astype(np.float32)
    ps = T.DevicePowerSpectrum(nb, 1.0, data=_dev(s))
    sums = T.HarmonicSums(ps, nfolds)
    T.HarmonicFolder(sums).fold(ps)
    want = oracle.harmonic_sums(s.astype(np.float64), nfolds)
    for h in range(nfolds):
        assert err_vs_rms(_host(sums[h].data), want[h]) < 1e-5


def test_harmonic_sums_vs_reference(T, ref_gpu):
    rng = np.random.default_rng(12)
    nb = (1 << 18) + 1
    s = rng.standard_normal(nb).astype(np.float32)
    ps = T.DevicePowerSpectrum(nb, 1.0, data=_dev(s))
    sums = T.HarmonicSums(ps, 5)
    T.HarmonicFolder(sums).fold(ps)
    want = ref_gpu.ref_harmonic_sums(s, 5)
    for h in range(5):
        got = _host(sums[h].data)
        assert np.array_equal(got, want[h]), f"fold {h + 1}: {np.count_nonzero(got != want[h])}"


def test_peak_finder_vs_oracle_and_reference(T, oracle):
    rng = np.random.default_rng(13)
    nb = (1 << 15) + 1
    spec = rng.standard_normal(nb).astype(np.float32)
    for c in (100, 101, 140, 175, 3000, 3020, 3051, 9000, 20000, 32700):
        spec[c] = 12.0 + (c % 7)
    spec[3010] = 13.5
    bw = float(np.float32(1.0 / np.float32(np.float32(1 << 16) * TS)))
    pf = T.PeakFinder(7.0, 0.1, 1100.0, 1 << 16)
    for nh in range(6):
        ps = T.DevicePowerSpectrum(nb, bw, nh, data=_dev(spec))
        sc = T.SpectrumCandidates(0.0, 0, 0.0)
        pf.find_candidates(ps, sc)
        got = np.array([(c.snr, c.freq) for c in sc.cands], np.float32).reshape(-1, 2)
        oi, osn, ofr = oracle.find_peaks(spec.astype(np.float64), bw, nh, 7.0, 0.1, 1100.0)
        assert np.array_equal(got[:, 1], ofr), nh
        assert np.allclose(got[:, 0], osn, rtol=1e-6)
        if os.path.exists(oracle.REF_GPU_PATH):
            rs, rf = oracle.ref_find_candidates(spec, bw, nh, 7.0, 0.1, 1100.0)
            assert np.array_equal(got[:, 0], rs) and np.array_equal(got[:, 1], rf), nh


def test_batched_resample_matches_single(psx, cuda):
    import ctypes as C
    torch = cuda
    n = 1 << 18
    x = torch.randn(n, device="cuda")
    accs = np.array([-50.0, -3.0, 0.0, 7.5, 99.0], np.float32)
    out = torch.empty((accs.size, n), device="cuda")
    assert psx.psx_resampleII_batch(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), n,
                                    accs.ctypes.data, accs.size, float(TS), None) == 0
    one = torch.empty(n, device="cuda")
    for t, a in enumerate(accs):
        assert psx.psx_resampleII(C.c_void_p(x.data_ptr()), C.c_void_p(one.data_ptr()), n,
                                  float(a), float(TS), None) == 0
        assert torch.equal(one, out[t])


@pytest.mark.parametrize("dtype", [np.uint8, np.int8])
@pytest.mark.parametrize("n", [1, 1000, (1 << 20) + 3])
def test_convert_8bit_vs_reference(T, psx, ref_gpu, dtype, n):
    """psx_convert_u8_f32 / psx_convert_i8_f32 (the conversion after the
    host->device copy of 8-bit series) against numpy's cast and against the
    reference's own ReusableDeviceTimeSeries::copy_from_host
    (conversion_kernel, src/kernels.cu:1171-1200): exact, the edge values
    0, 127, -128 (int8) and 255 (uint8) included."""
    import ctypes as C
    import torch
    rng = np.random.default_rng(n)
    info = np.iinfo(dtype)
    x = rng.integers(info.min, int(info.max) + 1, n, dtype=np.int64).astype(dtype)
    edges = np.array([0, 127, info.min, info.max, 1, info.max - 1], np.int64).astype(dtype)
    x[:min(n, edges.size)] = edges[:min(n, edges.size)]
    d_in = _dev(x)
    d_out = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
    fn = psx.psx_convert_u8_f32 if dtype == np.uint8 else psx.psx_convert_i8_f32
    rc = fn(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), C.c_size_t(n),
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, psx.psx_last_error()
    got = _host(d_out)
    assert np.array_equal(got, x.astype(np.float32))
    assert np.array_equal(got, ref_gpu.ref_copy_from_host_8bit(x))
