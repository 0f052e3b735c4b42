"""The product's host-side search logic (in libpeasoup_b200.so, called
through the C ABI on the CPU) against the oracle and the reference's own
host classes: acceleration plan, peak ranges, clustering, distillers."""
import ctypes as C
import os

import numpy as np
import pytest

from peasoup_b200 import _lib
from peasoup_b200 import transforms as T

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def hg():
    return np.load(os.path.join(GOLD, "host_golden.npz"))


def test_accel_list_against_golden(psx, hg):
    a = hg["overview_args"]
    plan = T.AccelerationPlan(a[0], a[1], a[2], a[3], int(hg["overview_nsamps"]), a[4], a[5], a[6])
    assert np.array_equal(plan.generate_accel_list(54.5, 54.5), hg["overview_accels"])
    cases, vals = hg["accel_cases"], hg["accel_values"]
    for ci, dm, off, n in hg["accel_index"]:
        c = cases[int(ci)]
        plan = T.AccelerationPlan(c[0], c[1], c[2], c[3], int(c[4]), c[5], c[6], c[7])
        got = plan.generate_accel_list(float(dm), float(c[8]))
        assert np.array_equal(got, vals[int(off):int(off) + int(n)]), (c, dm)


def test_accel_list_edge_cases(psx, oracle):
    plan = T.AccelerationPlan(5.0, 5.0, 1.1, 64e-6, 1 << 20, 64e-6, 1.4e9, 1e6)
    assert list(plan.generate_accel_list(0.0, 0.0)) == [5.0]
    plan = T.AccelerationPlan(10.0, 20.0, 1.1, 64e-6, 1 << 20, 64e-6, 1.4e9, 1e6)
    got = plan.generate_accel_list(3.0, 0.0)
    assert 0.0 not in got and got[0] == 10.0 and got[-1] == 20.0
    assert np.array_equal(got, oracle.accel_list(10.0, 20.0, 1.1, 64e-6, 1 << 20, 64e-6, 1.4e9,
                                                 1e6, 3.0, 0.0))


def test_peak_range_matches_oracle(psx, oracle):
    for n in (1 << 16, 3 << 18, 1 << 23, 1 << 27):
        for ts in (64e-6, 76e-6):
            tobs = np.float32(np.float32(n) * np.float32(ts))
            bw = float(np.float32(1.0 / tobs))
            for nh in range(6):
                s, e, f = C.c_int(), C.c_int(), C.c_float()
                psx.psx_peak_range(n // 2 + 1, bw, nh, 0.1, 1100.0, C.byref(s), C.byref(e),
                                   C.byref(f))
                assert (s.value, e.value, np.float32(f.value)) == tuple(
                    [*oracle.peak_range(n // 2 + 1, bw, nh, 0.1, 1100.0)[:2],
                     np.float32(oracle.peak_range(n // 2 + 1, bw, nh, 0.1, 1100.0)[2])])


def test_unique_peaks_matches_oracle(psx, oracle):
    rng = np.random.default_rng(0)
    for _ in range(50):
        k = int(rng.integers(1, 400))
        idx = np.sort(rng.choice(20000, size=k, replace=False)).astype(np.int32)
        snr = rng.uniform(7, 30, size=k).astype(np.float32)
        oi = np.zeros(k, np.int32)
        os_ = np.zeros(k, np.float32)
        n = psx.psx_identify_unique_peaks(idx.ctypes.data, snr.ctypes.data, k, 30,
                                          oi.ctypes.data, os_.ctypes.data)
        pi, ps = oracle.identify_unique_peaks(idx, snr.astype(np.float64), 30)
        assert np.array_equal(oi[:n], pi)
        assert np.array_equal(os_[:n], ps.astype(np.float32))


@pytest.mark.parametrize("name,kind", [("harm", 0), ("harm_related", 0), ("accel", 1), ("dm", 2)])
def test_distillers_match_reference_golden(psx, hg, name, kind):
    for j in range(4):
        c = np.ascontiguousarray(hg[f"distill_{name}_{j}_in"]).copy()
        want = hg[f"distill_{name}_{j}_out"]
        wna = hg[f"distill_{name}_{j}_nassoc"]
        na = np.zeros(max(1, c.size), np.int32)
        kw = {"harm": (1e-4, 16.0, 0.0, 0, 1), "harm_related": (1e-4, 16.0, 0.0, 1, 0),
              "accel": (1e-4, 16.0, 637.5, 1, 1), "dm": (1e-4, 16.0, 0.0, 1, 1)}[name]
        n = psx.psx_distill(kind, c.ctypes.data, c.size, *kw, na.ctypes.data)
        assert np.array_equal(c[:n], want), (name, j)
        assert np.array_equal(na[:n], wna), (name, j)


def test_harmonic_distiller_fast_path_equals_exhaustive(psx, oracle):
    """The product tests only the few kk near jj*f0/f for each jj; the
    oracle runs the reference's exhaustive double loop."""
    rng = np.random.default_rng(5)
    for trial in range(20):
        n = int(rng.integers(2, 200))
        f0 = rng.uniform(1, 300, size=5)
        c = np.zeros(n, oracle.CAND_DTYPE)
        for i in range(n):
            b = f0[rng.integers(5)]
            freq = b * rng.integers(1, 20) / 2 ** rng.integers(0, 6) * (1 + rng.normal(0, 5e-5))
            c[i] = (1.0, 0, 0.0, rng.integers(0, 6), rng.uniform(6, 50), freq)
        mine = c.copy()
        na = np.zeros(n, np.int32)
        k = psx.psx_distill(0, mine.ctypes.data, n, 1e-4, 16.0, 0.0, 1, 1, na.ctypes.data)
        surv, arr, keep, ona = oracle.harmonic_distill(c, 1e-4, 16.0, True)
        assert np.array_equal(mine[:k], surv)
        assert np.array_equal(na[:k], ona[keep == 1])


def test_distillers_live_reference(ref_host, psx):
    rng = np.random.default_rng(9)
    for trial in range(10):
        n = int(rng.integers(2, 120))
        c = np.zeros(n, ref_host.CAND_DTYPE)
        for i in range(n):
            c[i] = (2.0, 1, rng.choice([-20.0, 0.0, 20.0]), rng.integers(0, 6),
                    rng.uniform(6, 20), rng.choice([50.0, 100.0, 25.0, 33.3333]) *
                    (1 + rng.normal(0, 1e-4)))
        for kind, kw in ((0, dict(keep_related=True, fractional=True)),
                         (1, dict(tobs=300.0, keep_related=True)),
                         (2, dict(keep_related=True))):
            want, wna = ref_host.ref_distill(kind, c, **kw)
            mine = c.copy()
            na = np.zeros(n, np.int32)
            k = psx.psx_distill(kind, mine.ctypes.data, n, 1e-4, 16.0, kw.get("tobs", 0.0),
                                1, int(kw.get("fractional", True)), na.ctypes.data)
            assert np.array_equal(mine[:k], want), kind
            assert np.array_equal(na[:k], wna), kind
