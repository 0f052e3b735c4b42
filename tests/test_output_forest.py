"""The post-search chain on candidate forests against the reference's own
host code (built from its sources into oracle/_ref): the distillers with
association trees (global DMDistiller and HarmonicDistiller), the
CandidateScorer, candidates.peasoup and overview.xml.  CPU only."""
import os
import tempfile

import numpy as np
import pytest

from peasoup_b200 import _lib, output
from peasoup_b200.search import CAND_DTYPE

TSAMP, CFREQ, FOFF, BW = 64e-6, 1475.12, -1.09, 69.76   # MHz, as the reference passes them


def _dm_lists(seed, ndm=12):
    """Per-DM candidate lists shaped like a search's: a few pulsars seen at
    several DM trials, accelerations and harmonics, plus noise peaks; S/N
    with deliberate ties."""
    rng = np.random.default_rng(seed)
    f0s = rng.uniform(2.0, 400.0, 4)
    out = []
    for d in range(ndm):
        rows = []
        for f0 in f0s:
            for h in (1, 2, 3, 0.5):
                if rng.uniform() < 0.6:
                    # the same signal at one to three acceleration trials
                    for acc in rng.choice([-20.0, 0.0, 5.5, 20.0], int(rng.integers(1, 4)),
                                          replace=False):
                        rows.append((0.5 * d, d, float(acc), int(rng.integers(0, 5)),
                                     float(np.round(rng.uniform(7, 30), 1)),
                                     float(f0 * h * (1 + rng.normal(0, 2e-5)))))
        for _ in range(int(rng.integers(2, 8))):
            rows.append((0.5 * d, d, float(rng.uniform(-50, 50)), int(rng.integers(0, 5)),
                         float(np.round(rng.uniform(7, 12), 1)), float(rng.uniform(0.1, 1000))))
        out.append(np.array(rows, CAND_DTYPE))
    return out


def _per_dm_forests(ref, lists, tobs, tol=1e-4):
    """The Worker's per-DM AccelerationDistiller (keep_related) by the
    product, checked against the reference on the way."""
    forests = []
    for c in lists:
        leaves = output.leaves(c)
        got = output.distill_forest(_lib.PSX_DISTILL_ACCEL, *leaves, tol=tol, tobs=tobs,
                                    keep_related=True, fractional=True)
        want = ref.ref_distill_forest(1, *leaves, tol=tol, tobs=tobs, keep_related=True,
                                      fractional=True)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
        forests.append(got)
    return forests


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_forest_distillation_matches_reference(ref_host, seed):
    ref = ref_host
    tobs = float(np.float32((1 << 20) * TSAMP))
    forests = _per_dm_forests(ref, _dm_lists(seed), tobs)
    nodes, sizes = output.concat(forests)
    assert (sizes > 1).any()
    for kind, fr in ((_lib.PSX_DISTILL_DM, False), (_lib.PSX_DISTILL_HARMONIC, False),
                     (_lib.PSX_DISTILL_HARMONIC, True), (_lib.PSX_DISTILL_ACCEL, True)):
        for keep in (True, False):
            got = output.distill_forest(kind, nodes, sizes, tol=1e-4, max_harm=16.0, tobs=tobs,
                                        keep_related=keep, fractional=fr)
            want = ref.ref_distill_forest(kind, nodes, sizes, tol=1e-4, max_harm=16.0, tobs=tobs,
                                          keep_related=keep, fractional=fr)
            assert np.array_equal(got[0], want[0]), (kind, fr, keep)
            assert np.array_equal(got[1], want[1]), (kind, fr, keep)
    # the reference's chain after the Workers: DM, then harmonics (trees kept)
    n1, s1 = output.distill_forest(_lib.PSX_DISTILL_DM, nodes, sizes, keep_related=True)
    n2, s2 = output.distill_forest(_lib.PSX_DISTILL_HARMONIC, n1, s1, keep_related=True)
    r1 = ref.ref_distill_forest(2, nodes, sizes, keep_related=True)
    r2 = ref.ref_distill_forest(0, *r1, keep_related=True, fractional=False)
    assert np.array_equal(n2, r2[0]) and np.array_equal(s2, r2[1])
    assert (s2 > 2).any()   # trees of depth > 1 came through


def test_scores_match_reference(ref_host):
    ref = ref_host
    tobs = float(np.float32((1 << 20) * TSAMP))
    nodes, sizes = output.concat(_per_dm_forests(ref, _dm_lists(7, ndm=20), tobs))
    nodes, sizes = output.distill_forest(_lib.PSX_DISTILL_DM, nodes, sizes, keep_related=True)
    got = output.score_forest(nodes, sizes, TSAMP, CFREQ, FOFF, BW)
    want = ref.ref_score_forest(nodes, sizes, TSAMP, CFREQ, FOFF, BW)
    assert len(got) == len(want) > 5
    assert got.tobytes() == want.tobytes()
    assert got["is_adjacent"].any() and (got["ddm_count_ratio"] < 1).any()


def test_candidate_file_and_overview_match_reference(ref_host):
    ref = ref_host
    tobs = float(np.float32((1 << 20) * TSAMP))
    nodes, sizes = output.concat(_per_dm_forests(ref, _dm_lists(9), tobs))
    nodes, sizes = output.distill_forest(_lib.PSX_DISTILL_DM, nodes, sizes, keep_related=True)
    with tempfile.TemporaryDirectory() as d:
        off = output.write_candidates(os.path.join(d, "mine.peasoup"), nodes, sizes)
        # the reference resolves the path with realpath() before opening it,
        # so its file must exist already (output_stats.hpp:278-281)
        open(os.path.join(d, "ref.peasoup"), "wb").close()
        roff = ref.ref_write_binary(d, "ref.peasoup", nodes, sizes)
        mine = open(os.path.join(d, "mine.peasoup"), "rb").read()
        theirs = open(os.path.join(d, "ref.peasoup"), "rb").read()
    assert mine == theirs and np.array_equal(off, roff)
    # read back as the reference's tools do (tools/peasoup_tools.py)
    r = output.roots(sizes)
    first = np.frombuffer(mine, np.int32, count=1, offset=int(off[1]))[0]
    assert first == sizes[r[1]]
    dms = (0.5 * np.arange(12)).astype(np.float32)
    accs = np.array([-20.0, -3.3333333, 0.0, 5.5, 20.0], np.float32)
    scores = output.score_forest(nodes, sizes, TSAMP, CFREQ, FOFF, BW)
    text = (output.Overview().dm_list(dms).acc_list(accs, 0.0)
            .candidates(nodes, sizes, scores, off).text())
    want = ref.ref_overview_text(dms, accs, 0.0, nodes, sizes, off, TSAMP, CFREQ, FOFF, BW)
    assert text == want


def test_forest_sizes_are_validated(psx):
    import ctypes as C
    nodes = np.zeros(3, CAND_DTYPE)
    bad = np.array([2, 2, 1], np.int32)    # the child runs past its parent
    n, nr = C.c_size_t(), C.c_size_t()
    rc = psx.psx_distill_forest(0, nodes.ctypes.data, bad.ctypes.data, 3, 1e-4, 16.0, 0.0, 1, 0,
                                None, None, 0, C.byref(n), C.byref(nr))
    assert rc == _lib.PSX_ERR_INVALID


def test_cpp_dropin_post_chain_matches_reference(ref_host):
    """tests/cpp/dropin_post.cpp (the drop-in C++ classes, compiled here)
    against the reference's own classes on the same per-DM forests."""
    import subprocess
    ref = ref_host
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    tobs = float(np.float32((1 << 20) * TSAMP))
    forests = _per_dm_forests(ref, _dm_lists(11, ndm=16), tobs)
    limit = 25
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "dropin_post")
        r = subprocess.run(["g++", "-O2", "-std=c++17", f"-I{root}/include",
                            "-I/usr/local/cuda/include", f"{root}/tests/cpp/dropin_post.cpp",
                            f"-L{root}/peasoup_b200", "-lpeasoup_b200", "-L/usr/local/cuda/lib64",
                            "-lcudart", f"-Wl,-rpath,{root}/peasoup_b200", "-o", exe],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        inp = os.path.join(d, "in.bin")
        with open(inp, "wb") as f:
            np.array([len(forests)], np.int32).tofile(f)
            for nodes, sizes in forests:
                np.array([len(nodes)], np.int32).tofile(f)
                np.ascontiguousarray(nodes, CAND_DTYPE).tofile(f)
                np.ascontiguousarray(sizes, np.int32).tofile(f)
        out = os.path.join(d, "mine")
        r = subprocess.run([exe, inp, out, str(limit), repr(TSAMP), repr(CFREQ), repr(FOFF),
                            repr(BW)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        nodes, sizes = output.concat(forests)
        r1 = ref.ref_distill_forest(2, nodes, sizes, keep_related=True)
        rn, rs = ref.ref_distill_forest(0, *r1, keep_related=True, fractional=False)
        rn, rs = output.limit(rn, rs, limit)
        assert int(r.stdout) == len(output.roots(rs)) == limit
        open(os.path.join(d, "ref.peasoup"), "wb").close()
        off = ref.ref_write_binary(d, "ref.peasoup", rn, rs)
        assert (open(os.path.join(out, "candidates.peasoup"), "rb").read() ==
                open(os.path.join(d, "ref.peasoup"), "rb").read())
        want = ref.ref_overview_text((0.5 * np.arange(16)).astype(np.float32),
                                     np.zeros(1, np.float32), 0.0, rn, rs, off, TSAMP, CFREQ,
                                     FOFF, BW)
        assert open(os.path.join(out, "overview.xml"), encoding="latin-1").read() == want
