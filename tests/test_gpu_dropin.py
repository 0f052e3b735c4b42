"""The C++ drop-in classes (include/transforms, utils, data_types) driven
in the reference's DM-loop call order (tests/cpp/dropin_pipeline.cpp,
compiled here with g++ against libpeasoup_b200.so) find exactly the
candidates of the fused engine's plain schedule on the same series."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def dropin_exe(psx, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "dropin_pipeline")
    cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT}/include", "-I/usr/local/cuda/include",
           f"{ROOT}/tests/cpp/dropin_pipeline.cpp", f"-L{ROOT}/peasoup_b200", "-lpeasoup_b200",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{ROOT}/peasoup_b200", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("case", ["white", "padded_zapped"])
def test_dropin_pipeline_matches_engine(cuda, dropin_exe, tmp_path, case):
    from peasoup_b200 import search, synth
    from peasoup_b200.search import CAND_DTYPE
    ts = 64e-6 if case == "white" else 76e-6
    n = 1 << 16
    if case == "white":
        x = synth.make_series_np(synth.SeriesSpec(
            nsamps=n, tsamp=ts, pulsars=[synth.Pulsar(5.7e-3, 12.0, 0.05, 1.0)]), 0)
        nsamps, zap, bf, bw = n, "-", np.zeros(0, np.float32), np.zeros(0, np.float32)
        kw = dict(acc_lo=-50.0, acc_hi=50.0, nharmonics=4, min_snr=7.0)
    else:
        plan = synth.survey_plan(ndm=1, nsamps=n - 1000, tsamp=ts, seed=3, npulsars=1, nbirdies=5)
        plan.pulsars[0].amp = 40.0
        x = synth.survey_series_np(plan, 0, seed=3)
        nsamps = x.size
        zap = str(tmp_path / "zap.txt")
        open(zap, "w").write(plan.zaplist_text())
        bf, bw = plan.birdie_freqs, plan.birdie_widths
        kw = dict(acc_lo=-100.0, acc_hi=100.0, nharmonics=5, min_snr=6.0)
    sp = str(tmp_path / "series.f32")
    x.astype(np.float32).tofile(sp)
    out = str(tmp_path / "cands.bin")
    r = subprocess.run([dropin_exe, sp, str(nsamps), str(n), repr(ts), "0", str(kw["acc_lo"]),
                        str(kw["acc_hi"]), str(kw["nharmonics"]), str(kw["min_snr"]), zap, out],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=CAND_DTYPE)
    s = search.AccelSearch(search.SearchParams(
        fft_size=n, tsamp=ts, cfreq_hz=1475.12e6, ch_bw_hz=1.09e6, mode="plain",
        birdie_freqs=bf, birdie_widths=bw, **kw))
    want = s.search(x, 0.0, 0, per_dm=True)[0]
    s.close()
    assert len(want) > 0
    assert np.array_equal(got, want)
