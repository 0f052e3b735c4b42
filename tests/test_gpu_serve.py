"""The served loop (psx_server, C++): requests of uneven transform length,
DM count and acceleration range admitted as they arrive and searched
concurrently.  Each result must be exactly what the same request gives
alone, on a fresh search instance, and on a retargeted pooled instance."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [1 << 16, 3 << 15, 1 << 17, 1 << 16, 3 << 16, 1 << 17]


@pytest.fixture(scope="module")
def M(cuda, psx):
    from peasoup_b200 import search, serve, synth
    return search, serve, synth


def _requests(M):
    search, serve, synth = M
    rng = np.random.default_rng(11)
    reqs = []
    for i, n in enumerate(SIZES):
        ndm = 2 + i % 3
        ts = 64e-6
        xs = np.stack([synth.make_series_np(synth.SeriesSpec(
            nsamps=n, tsamp=ts, pulsars=[synth.Pulsar(float(rng.uniform(2e-3, 9e-3)),
                                                      float(rng.uniform(-40, 40)), 0.05, 0.7)]),
            100 * i + d) for d in range(ndm)])
        acc = float(rng.uniform(20, 120))
        p = search.SearchParams(fft_size=n, tsamp=ts, acc_lo=-acc, acc_hi=acc,
                                nharmonics=3 + i % 3, min_snr=6.0, cfreq_hz=synth.CFREQ_HZ,
                                ch_bw_hz=synth.CH_BW_HZ)
        dms = (0.5 * np.arange(ndm)).astype(np.float32)
        reqs.append((p, xs, dms))
    return reqs


def _alone(M, p, xs, dms):
    search = M[0]
    s = search.AccelSearch(p)
    c, na, tr, dm = s.search_block(xs, dms)
    s.close()
    return c, na, dm


@pytest.mark.parametrize("policy", ["least_work", "even", "exclusive"])
def test_mixed_equals_alone(M, policy):
    search, serve, synth = M
    import torch
    reqs = _requests(M)
    srv = serve.Server(40 << 30, max_active=3, policy=policy)
    # half of the requests from device memory, half from host memory
    tickets = []
    for i, (p, xs, dms) in enumerate(reqs):
        src = torch.from_numpy(xs).cuda() if i % 2 else xs
        tickets.append(srv.submit(p, src, dms))
    got = [srv.wait(t) for t in tickets]
    st = srv.status()
    assert st["active"] == 0 and st["pending"] == 0 and st["pooled"] >= 1
    srv.close()
    if policy == "exclusive":  # one request on the device at a time
        spans = sorted((g[3]["t_admit"], g[3]["t_done"]) for g in got)
        assert all(b[0] >= a[1] for a, b in zip(spans, spans[1:])), spans
    for (p, xs, dms), (c, na, dm, stats) in zip(reqs, got):
        assert stats["status"] == 0 and stats["ndm"] == len(dms) and stats["ntrials"] > 0
        assert stats["t_submit"] <= stats["t_admit"] <= stats["t_done"]
        ac, ana, adm = _alone(M, p, xs, dms)
        assert len(c) > 0
        assert np.array_equal(c, ac) and np.array_equal(na, ana) and np.array_equal(dm, adm)


def test_pooled_instance_is_retargeted(M):
    """Two requests with the same instance shape but different acceleration
    ranges, fold counts, tsamp-derived limits and birdies: the second reuses
    the pooled instance and must still equal a fresh instance's result."""
    search, serve, synth = M
    import dataclasses
    reqs = _requests(M)
    p, xs, dms = reqs[0]
    p2 = dataclasses.replace(p, acc_lo=-75.0, acc_hi=60.0, min_snr=5.5, max_freq=900.0,
                             nharmonics=3 if p.nharmonics != 3 else 5,
                             birdie_freqs=np.array([50.0, 120.0], np.float32),
                             birdie_widths=np.array([0.3, 0.5], np.float32))
    srv = serve.Server(40 << 30, max_active=1)
    c1, _, _, s1 = srv.wait(srv.submit(p, xs, dms))
    c2, na2, dm2, s2 = srv.wait(srv.submit(p2, xs, dms))
    srv.close()
    assert s1["engine_reused"] == 0 and s1["footprint"] > 0
    assert s2["engine_reused"] == 1 and s2["footprint"] == 0
    a2, ana2, adm2 = _alone(M, p2, xs, dms)
    assert np.array_equal(c2, a2) and np.array_equal(na2, ana2)
    assert np.array_equal(c1, _alone(M, p, xs, dms)[0])


def test_admission_limits(M):
    search, serve, synth = M
    from peasoup_b200 import _lib
    from peasoup_b200._lib import PsxError
    reqs = _requests(M)
    p, xs, dms = reqs[2]
    need = search.footprint(p)
    # larger than the whole budget: refused at submission
    srv = serve.Server(need // 2, max_active=1)
    with pytest.raises(PsxError) as e:
        srv.submit(p, xs, dms)
    assert e.value.status == _lib.PSX_ERR_ALLOC
    srv.close()
    # one slot, a queue of one: a burst of four must see the queue full
    srv = serve.Server(need * 2, max_active=1, max_queue=1)
    ok, busy = [], 0
    for _ in range(4):
        try:
            ok.append(srv.submit(p, xs, dms))
        except PsxError as ex:
            assert ex.status == _lib.PSX_ERR_BUSY
            busy += 1
    assert busy >= 1 and len(ok) >= 1
    first = None
    for t in ok:
        c, na, dm, st = srv.wait(t)
        assert st["status"] == 0
        first = c if first is None else first
        assert np.array_equal(c, first)
    srv.close()


def test_exclusive_order_and_no_starvation(M):
    """PSX_SERVE_EXCLUSIVE admits the pending request with the least work,
    but a request passed over 8 times goes next: behind a running blocker,
    a long request L and ten short ones queue; the short ones go first
    until L has been passed over 8 times, then L, then the last two."""
    search, serve, synth = M
    ts = 64e-6

    import torch
    g = torch.Generator(device="cuda").manual_seed(5)

    def req(n, ndm, acc):  # white noise on the device
        xs = torch.randn((ndm, n), device="cuda", generator=g)
        p = search.SearchParams(fft_size=n, tsamp=ts, acc_lo=-acc, acc_hi=acc, nharmonics=3,
                                min_snr=8.0, cfreq_hz=synth.CFREQ_HZ, ch_bw_hz=synth.CH_BW_HZ)
        return p, xs, (0.5 * np.arange(ndm)).astype(np.float32)

    blocker = req(1 << 22, 48, 300.0)
    long_ = req(1 << 18, 16, 200.0)
    shorts = [req(1 << 16, 2, 20.0) for _ in range(10)]
    torch.cuda.synchronize()
    srv = serve.Server(40 << 30, max_active=2, policy="exclusive")
    tb = srv.submit(*blocker)
    tl = srv.submit(*long_)
    ts_ = [srv.submit(*r) for r in shorts]
    sb = srv.wait(tb)[3]
    sl = srv.wait(tl)[3]
    ss = [srv.wait(t)[3] for t in ts_]
    srv.close()
    assert all(s["status"] == 0 for s in [sb, sl] + ss)
    # the queue formed while the blocker ran
    assert sl["t_submit"] < sb["t_done"] and max(s["t_submit"] for s in ss) < sb["t_done"]
    order = sorted([("L", sl["t_admit"])] + [("S", s["t_admit"]) for s in ss],
                   key=lambda x: x[1])
    assert [o[0] for o in order] == ["S"] * 8 + ["L"] + ["S"] * 2, order
    spans = sorted((s["t_admit"], s["t_done"]) for s in [sb, sl] + ss)
    assert all(b[0] >= a[1] for a, b in zip(spans, spans[1:]))
