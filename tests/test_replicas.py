"""DM-sharded replicas on CPU: two gloo ranks each search their own DM
trials (with the CPU oracle standing in for the per-rank search) and
gather the candidate lists on the host; the gathered result must equal a
single-process search of every DM."""
import os
import socket

import numpy as np
import pytest

from peasoup_b200 import replicas


def test_partition_covers_each_dm_once():
    for ndm in (1, 7, 256, 257):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                seen += replicas.dm_partition(ndm, r, world, 8)
            assert sorted(seen) == list(range(ndm))


def test_schedule_is_rank_disjoint_within_a_pass():
    sched = [replicas.dm_schedule(256, r, 4, 8, 8) for r in range(4)]
    flat = [d for s in sched for st in s for d in st]
    assert len(flat) == len(set(flat)) == 256


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _series(d, n):
    from peasoup_b200 import synth
    return synth.make_series_np(synth.SeriesSpec(
        nsamps=n, tsamp=64e-6, pulsars=[synth.Pulsar(3e-3 * (1 + d), 5.0 * d, 0.05, 1.2)]), d)


def _search(oracle, d, n):
    from peasoup_b200 import synth
    p = oracle.SearchParams(fft_size=n, tsamp=64e-6, dm=0.5 * d, dm_idx=d, acc_lo=-20.0,
                            acc_hi=20.0, nharmonics=3, min_snr=7.0, cfreq=synth.CFREQ_HZ,
                            ch_bw=synth.CH_BW_HZ)
    c, _ = oracle.search_dm(_series(d, n), p)
    return c


def _rank_main(rank, world, port, ndm, n, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from oracle import oracle as O
    from peasoup_b200 import replicas as R
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = R.dm_partition(ndm, rank, world, 2)
        local = np.concatenate([_search(O, d, n) for d in mine]) if mine else \
            np.zeros(0, O.CAND_DTYPE)
        allc = R.gather_candidates(local)
        if rank == 0:
            np.save(out_path, allc)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_gather_equals_single_process(oracle, tmp_path):
    import torch.multiprocessing as mp
    ndm, n = 5, 1 << 14
    out = str(tmp_path / "gathered.npy")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, ndm, n, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    got = np.load(out)
    want = np.concatenate([_search(oracle, d, n) for d in range(ndm)])
    assert np.array_equal(got, want)
    assert len(want) > 0
