#!/usr/bin/env python
"""Benchmark of the per-DM acceleration search (Peasoup's hot loop) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl psx|reference]

Workload (the survey-shape configuration the headline metric is quoted on):
256 DM trials x 2^23 float32 samples, tsamp 76 us, uint8-quantised noise
(mean 128, sigma 20) with 1/f^1.5 red noise below 1 Hz, 5 injected
accelerated pulsars, 20 birdies injected and zapped, acceleration range
-100..100 m/s^2 at the default tolerance, 5 harmonic folds, S/N threshold 9
(the reference's default).  Data are seeded synthetic series made on the
GPU (no survey data offline).  A step searches `--dms-per-step` DM trials
(prologue + every acceleration trial + candidate distillation); K steps
cover K*S DM trials of the 256 (weak scaling over ranks: rank r takes its
own DM trials).  Every step's series (8 x 32 MB) exceed L2.

Printed: one JSON line.  `value` = DM x acceleration trials per second of
the batched path with the series resident in HBM; `e2e` = the same through
the C ABI (psx_search_block) from pinned host buffers (host->device copies
inside the timed region, candidates copied back); `plain` = the one-trial-
per-launch path on a sample of the same workload; `served` = the served
workload (Poisson arrivals of uneven segmented searches through the C++
server, p50/p95/p99 latency from arrival and from admission, each request
also run alone for the ratios); `roofline` = the
dominant stage's achieved HBM bytes/s against the measured copy bandwidth;
`cpu_baseline` = an FP32 C++ rendering of the same stages (MKL FFT through
libtorch) on one whole DM trial, on every host core.

`--impl reference` times the reference's own implementation of the path
(its src/kernels.cu, transforms and unmodified Worker::start, built for
sm_100a into oracle/_ref) over the same DM trials of the same series, one
Worker for the whole list as the reference's program runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DM×accel trials/s at 2^23 pts batched vs plain, %HBM roofline; served p50/p99"
N_FFT = 1 << 23
TSAMP = 76e-6
ACC = 100.0
NFOLDS = 5
NDM = 256
SERVED_REQUESTS = 32
FFT_FORMS = {1: "cuFFT complex transform + fused unpack/interbin/normalise",
             2: "cuFFT real transform + interbin/normalise (the reference's)",
             3: "two-pass transform with the resample gather in pass 1 + "
                "unpack/interbin/normalise"}
SERVED_TRIAL_BUDGET = 2000
SERVED_SLOTS = 2
SERVED_BUDGET = 150_000_000_000


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = str(index)
        try:
            import torch
            u = str(torch.cuda.get_device_properties(index).uuid)
            self.index = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            pass
        self.proc = None
        self.f = tempfile.TemporaryFile(mode="w+")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def dm_schedule(rank, ws, steps, per_step, offset=0):
    """DM indices of each step of this rank (rank-interleaved blocks)."""
    from peasoup_b200.replicas import dm_schedule as sched
    return sched(NDM, rank, ws, steps, per_step, offset)


def trials_of(plan, dm_list):
    from peasoup_b200 import synth
    from peasoup_b200.transforms import AccelerationPlan
    ap = AccelerationPlan(-ACC, ACC, 1.10, 64e-6, N_FFT, TSAMP, synth.CFREQ_HZ, synth.CH_BW_HZ)
    return sum(len(ap.generate_accel_list(float(plan.dms[d]), 0.0)) for d in dm_list)


def make_params(plan, mode="batched", batch=0, harm_shape=0):
    from peasoup_b200 import search, synth
    return search.SearchParams(fft_size=N_FFT, tsamp=TSAMP, acc_lo=-ACC, acc_hi=ACC,
                               nharmonics=NFOLDS, cfreq_hz=synth.CFREQ_HZ,
                               ch_bw_hz=synth.CH_BW_HZ, birdie_freqs=plan.birdie_freqs,
                               birdie_widths=plan.birdie_widths, mode=mode, batch=batch,
                               harm_shape=harm_shape)


# ----------------------------------------------------------------- reference
def _standalone(name):
    """peasoup_b200/<name>.py loaded as a module of its own, without the
    package (whose library the reference arm must not load).  Used for the
    pure numpy/torch modules: the synthetic workload and the DM schedule."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        f"_bench_{name}", os.path.join(ROOT, "peasoup_b200", f"{name}.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod   # dataclasses look their module up there
    spec.loader.exec_module(mod)
    return mod


def _mapped_native_libraries():
    """Shared libraries of this repository mapped into the process."""
    seen = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.startswith(ROOT) and ".so" in path:
                    seen.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(seen)


def run_reference(args, ws, rank):
    """The reference's own implementation of the path on the same workload:
    its src/kernels.cu, transform classes and unmodified Worker::start,
    built for sm_100a into oracle/_ref, over exactly the DM trials and
    series of the --impl psx arm's timed steps (same seeds, same schedule,
    same zap list).  As in the reference's program, one Worker searches the
    whole DM list (its set-up of plans and buffers once, then DM trial by
    DM trial, host->device copy of each series included); the time is that
    of Worker::start.  Trials are counted with the reference's own
    AccelerationPlan (oracle/_ref host build).  Nothing of this
    repository's library is loaded in this process."""
    if rank != 0:
        return 0
    from oracle import oracle as O
    if not (os.path.exists(O.REF_GPU_PATH) and os.path.exists(O.REF_HOST_PATH)):
        print(json.dumps({"impl": "reference", "metric": METRIC,
                          "unavailable": "oracle/_ref libraries not built "
                                         "(build() compiles them where the reference sources "
                                         "exist)"}), flush=True)
        return 0
    import ctypes as C
    import torch
    synth = _standalone("synth")
    repl = _standalone("replicas")
    S = args.dms_per_step
    plan = synth.survey_plan(ndm=NDM, nsamps=N_FFT, tsamp=TSAMP)
    # the schedule and the synthesis calls of the psx arm at one rank
    warm = repl.dm_schedule(NDM, 0, 1, args.warmup, S, args.steps)
    timed = repl.dm_schedule(NDM, 0, 1, args.steps, S)
    need = sorted({d for st in warm + timed for d in st})
    block = synth.survey_block_torch(plan, dm_indices=need)
    row = {d: i for i, d in enumerate(need)}
    p = O.SearchParams(fft_size=N_FFT, tsamp=TSAMP, acc_lo=-ACC, acc_hi=ACC, nharmonics=NFOLDS,
                       cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ)
    warm_dms = [d for st in warm for d in st]
    timed_dms = [d for st in timed for d in st]
    L = O.ref_gpu()
    L.ref_worker_search_timed.restype = C.c_int
    a = O._RefArgs(p.cdm, p.acc_lo, p.acc_hi, p.acc_tol, p.acc_pulse_width * 1e6, p.cfreq,
                   p.ch_bw, p.nharmonics, p.min_snr, p.min_freq, p.max_freq, int(p.max_harm),
                   p.freq_tol, b"")
    fd, zap = tempfile.mkstemp(suffix=".txt")
    with os.fdopen(fd, "w") as f:
        f.write(plan.zaplist_text())
    a.zapfile = zap.encode()

    def worker(dm_list):
        rows = torch.stack([block[row[d]] for d in dm_list]).cpu().numpy()
        cap = 1 << 20
        out = np.zeros(cap, O.CAND_DTYPE)
        na = np.zeros(cap, np.int32)
        n = C.c_size_t()
        sec = C.c_double()
        dms = np.ascontiguousarray(plan.dms[dm_list], np.float32)
        rc = L.ref_worker_search_timed(rows.ctypes.data_as(C.c_void_p), C.c_size_t(len(dm_list)),
                                       C.c_size_t(N_FFT), C.c_float(TSAMP),
                                       dms.ctypes.data_as(C.c_void_p), C.c_size_t(N_FFT),
                                       C.byref(a), out.ctypes.data_as(C.c_void_p),
                                       na.ctypes.data_as(C.c_void_p), C.c_size_t(cap),
                                       C.byref(n), C.byref(sec))
        if rc != 0:
            raise RuntimeError(f"reference Worker failed with status {rc}")
        return sec.value, int(n.value)

    try:
        worker(warm_dms)
        torch.cuda.synchronize()
        dt, ncand = worker(timed_dms)
    finally:
        os.unlink(zap)
    ntr = 0
    for d in timed_dms:
        ntr += len(O.ref_accel_list(-ACC, ACC, 1.10, 64e-6, N_FFT, TSAMP, synth.CFREQ_HZ,
                                    synth.CH_BW_HZ, float(plan.dms[d]), 0.0))
    v = ntr / dt
    loaded = _mapped_native_libraries()
    sample = (f"{len(timed_dms)} DM trials of the survey workload ({ntr} acceleration trials; "
              f"the --impl psx arm's timed DM trials), the reference's kernels.cu + transforms + "
              f"unmodified Worker::start built for sm_100a, one host thread driving cuda:0 (the "
              f"reference has no CPU implementation of this path)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "trials/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "survey-2^23: 256 DM trials x 2^23 samples, tsamp 76us, "
                               "acc -100..100, 5 folds, S/N 9, 20 birdies zapped",
                   "dms_per_step": S, "dm_trials": timed_dms[:1] + timed_dms[-1:],
                   "same_config_as_psx_arm": True,
                   "l2": "inputs larger than L2 (32 MB series per DM trial)"},
        "trials": ntr, "candidates": ncand,
        "cpu_baseline": {"value": v, "unit": "trials/s", "cores": 1, "kind": "reference",
                         "runs_on": "cuda:0", "sample": sample},
        "e2e": {"value": v, "unit": "trials/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "native_libraries_loaded": loaded,
    }), flush=True)
    return 0


# ----------------------------------------------------------------- CPU baseline
def _cpu_workers():
    """Spawned processes for the dedispersion CPU sample: every core,
    bounded by memory (about 1.5 GB each) and by 32."""
    n = os.cpu_count() or 1
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) for l in f if l.startswith("MemAvailable")) * 1024
        n = min(n, max(1, int(avail // 1.5e9)))
    except (OSError, StopIteration, ValueError):
        pass
    return max(1, min(n, 32))


def _cpu_threads():
    """Host threads for the CPU baseline: every core, at most 64."""
    return max(1, min(os.cpu_count() or 1, 64))


def cpu_baseline(plan, block_row, dm):
    """The FP32 CPU rendering of the same stages (oracle/cpu_render.cpp:
    the per-trial loop in FP32 with libtorch's MKL-backed FFT, FFTW being
    absent here; trials spread over one thread per core) on one whole DM
    trial of the workload, every acceleration trial of it included.
    Returns (trials per second, threads, trials, seconds)."""
    from oracle import oracle as O
    from peasoup_b200 import synth
    p = O.SearchParams(fft_size=N_FFT, tsamp=TSAMP, dm=float(dm), acc_lo=-ACC, acc_hi=ACC,
                       nharmonics=NFOLDS, cfreq=synth.CFREQ_HZ, ch_bw=synth.CH_BW_HZ,
                       birdie_freqs=np.asarray(plan.birdie_freqs),
                       birdie_widths=np.asarray(plan.birdie_widths))
    ntr = len(O.accel_list(-ACC, ACC, 1.10, 64e-6, N_FFT, TSAMP, synth.CFREQ_HZ,
                           synth.CH_BW_HZ, float(dm), 0.0))
    threads = _cpu_threads()
    x = np.ascontiguousarray(block_row, np.float32)
    _, _, sec = O.cpu_search_dm(x, p, threads)
    return ntr / sec, threads, ntr, sec


# ----------------------------------------------------------------- served
def _pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q)) if len(v) else None


def _served_series(r, seed):
    """One request's block on the device: white N(0,1) noise plus one
    injected accelerated pulse train per DM trial (seeded)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn((r.ndm, r.fft_size), device="cuda", generator=g)
    n = torch.arange(r.fft_size, device="cuda", dtype=torch.float64)
    rng = np.random.default_rng(seed)
    for d in range(r.ndm):
        f0 = float(np.exp(rng.uniform(np.log(2.0), np.log(500.0))))
        a = float(rng.uniform(-0.8, 0.8)) * r.acc_half
        k = a * r.tsamp / (2.0 * 299792458.0)
        ph = torch.frac(f0 * r.tsamp * (n - k * n * (n - r.fft_size)))
        x[d] += (0.3 * torch.exp(-0.5 * ((ph - 0.5) / 0.02) ** 2)).float()
    return x


def run_served(nreq, rank, log_prefix, policy="exclusive", nslots=SERVED_SLOTS):
    """The served workload (Poisson arrivals, uneven requests) through the
    C++ server under two scheduling policies, and every request alone on a
    one-slot server before and after them: latency from arrival and from
    admission, throughput, and the ratios to the isolated runs."""
    import threading as th
    import torch
    from peasoup_b200 import serve
    reqs = serve.served_stream(nreq, seed=1, rate=4.0, trial_budget=SERVED_TRIAL_BUDGET)
    params = [serve.request_params(r) for r in reqs]
    # every request's series made on the device before the passes (they are
    # resident in HBM as the served workload says), unless that is too much
    total = sum(4 * r.ndm * r.fft_size for r in reqs)
    pre = total < 64e9
    series = [_served_series(r, 1000 + i) for i, r in enumerate(reqs)] if pre else None
    torch.cuda.synchronize()

    def warm(srv, max_active):
        # a server in service has its instances built: one DM trial per
        # transform length and slot before the pass (all fit the budget)
        if not pre:
            return
        first = {}
        for i, r in enumerate(reqs):
            first.setdefault(r.fft_size, i)
        for i in first.values():
            x = series[i][:1]
            tk = [srv.submit(params[i], x, np.zeros(1, np.float32)) for _ in range(max_active)]
            for t in tk:
                srv.wait(t)

    def one_pass(max_active, paced, pol=policy, burst=False):
        srv = serve.Server(SERVED_BUDGET, max_active=max_active, policy=pol)
        warm(srv, max_active)
        res = [None] * len(reqs)
        tickets = [None] * len(reqs)
        ready = [th.Event() for _ in reqs]

        def collect():
            for i in range(len(reqs)):
                ready[i].wait()
                res[i] = srv.wait(tickets[i])[3]

        ct = th.Thread(target=collect)
        ct.start()
        t_start = srv.clock()
        arrivals = []
        for i, r in enumerate(reqs):
            if pre:
                x = series[i]
            else:
                x = _served_series(r, 1000 + i)
                torch.cuda.current_stream().synchronize()   # this stream only
            if paced and not burst:
                delay = t_start + r.arrival - srv.clock()
                if delay > 0:
                    time.sleep(delay)
                arrivals.append(t_start + r.arrival)
            elif paced:  # every request at once: the schedule's capacity
                arrivals.append(srv.clock())
            tickets[i] = srv.submit(params[i], x, np.arange(r.ndm, dtype=np.float32) * 0.5)
            if not paced:
                arrivals.append(srv.clock())
                ready[i].set()
                while res[i] is None:   # alone: one request on the device at a time
                    time.sleep(0.001)
            else:
                ready[i].set()
            del x
        ct.join()
        srv.close()
        return res, arrivals

    # the requested policy, and the other scheduling of the same stream for
    # comparison (exclusive runs one request at a time; the sharing policies
    # admit nslots at once)
    other = "least_work" if policy == "exclusive" else "exclusive"
    slots = {p: 1 if p == "exclusive" else nslots for p in (policy, other)}
    # isolated latencies: every request alone, before and after the served
    # passes; each request's ratios use the faster of its two (the device's
    # clock under the power cap drifts over a run)
    alone0, _ = one_pass(1, False)
    runs = {p: one_pass(slots[p], True, p) for p in (policy, other)}
    # capacity under the requested policy: the same requests all at once
    burst, _ = one_pass(slots[policy], True, policy, burst=True)
    alone1, _ = one_pass(1, False)
    alone = alone0 + alone1
    del series
    iso0 = [1e3 * (s["t_done"] - s["t_admit"]) for s in alone0]
    iso1 = [1e3 * (s["t_done"] - s["t_admit"]) for s in alone1]
    iso = [min(a, b) for a, b in zip(iso0, iso1)]
    iso_spread = _pct([max(a, b) / min(a, b) for a, b in zip(iso0, iso1)], 50)

    def summary(pol):
        mixed, arr = runs[pol]
        trials = sum(s["ntrials"] for s in mixed)
        lat_arr = [1e3 * (s["t_done"] - a) for s, a in zip(mixed, arr)]
        lat_adm = [1e3 * (s["t_done"] - s["t_admit"]) for s in mixed]
        span = max(s["t_done"] for s in mixed) - min(arr)
        served_tps = trials / span
        isolated_tps = trials / (sum(iso) / 1e3)
        ratio = [a / b for a, b in zip(lat_adm, iso)]
        # from arrival: the time a request spends in the system over its
        # isolated time (queueing included)
        ratio_arr = [a / b for a, b in zip(lat_arr, iso)]
        failed = sum(1 for s in mixed + alone if s["status"] != 0)
        worst = sorted(range(len(reqs)), key=lambda i: -ratio[i])[:4]
        return {
            "requests": len(reqs), "failed": failed, "arrival_rate_per_s": 4.0,
            "trials": int(trials), "trials_per_s": served_tps,
            "latency_from_arrival_ms": {"p50": _pct(lat_arr, 50), "p95": _pct(lat_arr, 95),
                                        "p99": _pct(lat_arr, 99)},
            "latency_from_admission_ms": {"p50": _pct(lat_adm, 50), "p95": _pct(lat_adm, 95),
                                          "p99": _pct(lat_adm, 99)},
            "isolated_ms": {"p50": _pct(iso, 50), "p99": _pct(iso, 99),
                            "before_after_spread_p50": iso_spread},
            "p99_admitted_over_p99_isolated": _pct(lat_adm, 99) / _pct(iso, 99),
            "per_request_ratio_p99": _pct(ratio, 99),
            "per_request_ratio_p50": _pct(ratio, 50),
            "per_request_arrival_ratio_p50": _pct(ratio_arr, 50),
            "per_request_arrival_ratio_p99": _pct(ratio_arr, 99),
            "worst_ratio_requests": [
                {"fft_size": reqs[i].fft_size, "ndm": reqs[i].ndm, "trials": mixed[i]["ntrials"],
                 "admitted_ms": lat_adm[i], "isolated_ms": iso[i], "ratio": ratio[i]}
                for i in worst],
            "throughput_over_isolated_back_to_back": served_tps / isolated_tps,
            # isolated device time of the stream over its arrival span: below
            # 1 the stream does not keep the device busy, and the served
            # trials/s measures the arrivals rather than the capacity
            "offered_load_over_capacity": (sum(iso) / 1e3) / max(1e-9, max(arr) - min(arr)),
            "max_active": slots[pol], "policy": pol, "hbm_budget_gb": SERVED_BUDGET / 1e9,
            "engines_reused": int(sum(s["engine_reused"] for s in mixed)),
            "series": "made on the GPU before the passes" if pre else "made at each arrival",
            "warm_up": ("every server (served and isolated passes) first searches one DM "
                        "trial per transform length and slot, so its instances exist"
                        if pre else "none"),
            "workload": (f"{len(reqs)} requests, Poisson 4/s (seed 1), fft_size in 2^20..2^25 "
                         f"incl. 3*2^k, DM count log-uniform 16..512 cut to <= "
                         f"{SERVED_TRIAL_BUDGET} 2^23-equivalent trials per request, acc "
                         f"half-range 10..300, 3..5 folds, white noise + one pulsar per DM"),
        }
    out = summary(policy)
    out["compared_policy"] = summary(other)
    burst_span = max(s["t_done"] for s in burst) - min(s["t_submit"] for s in burst)
    burst_tps = sum(s["ntrials"] for s in burst) / burst_span
    out["burst"] = {
        "what": "the same requests submitted at once under the requested policy: the "
                "served loop's capacity",
        "trials_per_s": burst_tps,
        "over_isolated_back_to_back": burst_tps / (out["trials"] / (sum(iso) / 1e3)),
        "failed": sum(1 for s in burst if s["status"] != 0),
    }
    return out


# ----------------------------------------------------------------- configs 3, 5
def _pulse_block_torch(ndm, n, ts, seed, pulsar=(5.7e-3, 12.0, 0.05, 0.3), sigma=1.0):
    """White N(0, sigma^2) noise plus one accelerated Gaussian pulse train
    per row (the small benchmark's statistics), made on the GPU."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    out = torch.empty((ndm, n), dtype=torch.float32, device="cuda")
    i = torch.arange(n, device="cuda", dtype=torch.float64)
    P, acc, duty, amp = pulsar
    k = acc * ts / (2.0 * 299792458.0)
    phi = (i - k * i * (i - n)) * (ts / P)
    dd = phi - torch.round(phi)
    sig = duty / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    pulse = (amp * sigma * torch.exp(-0.5 * (dd / sig) ** 2)).float()
    del i, phi, dd
    for r in range(ndm):
        out[r] = sigma * torch.randn(n, generator=g, device="cuda") + pulse
    return out


def stage_roofline(prof, n, form_used, shape_used, peak, peak_kind, traffic_json=True,
                   sm_mhz=None):
    """Per-stage device time per trial (CUDA events around every launch
    group of a profiled run: prof from AccelSearch.profile) and each stage's
    algorithmic bytes per trial; the dominant stage's achieved HBM bytes/s
    against the measured copy bandwidth.  Algorithmic bytes per trial of N
    samples (B = N/2 + 1 bins): resample 8N (read + write the series), the
    transform 4N + 8B, forming and normalising 12B, the harmonic kernel 4B
    (the normalised spectrum read once); with the two-pass transform, pass 1
    8N (gather the series, write M complex) and pass 2 8N."""
    B = n // 2 + 1
    per_trial_bytes = {"resample": 8.0 * n, "fft": 4.0 * n + 8.0 * B, "form": 12.0 * B,
                       "harm": 4.0 * B}
    stage_kernels = {"resample": "k_resample", "fft": "cuFFT", "form": "k_unpack_form_norm",
                     "harm": "k_harm_rows" if shape_used >= 6 else "k_harm_tiles"}
    if form_used == 3:
        per_trial_bytes.update(resample=8.0 * n, fft=8.0 * n)
        stage_kernels.update(resample="k_fft4_cols (gather + column transforms)",
                             fft="k_fft4_rows (row transforms)", form="k_unpack_form_norm_t")
    stage_ms = {"resample": prof["resample_ms"], "fft": prof["fft_ms"],
                "form": prof["form_ms"], "harm": prof["harm_ms"]}
    trials_prof = max(1, prof["trials"])
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if traffic_json and os.path.exists(tp) and n == N_FFT:
        tj = json.load(open(tp))
        tkey = "harm_rows" if (dom == "harm" and shape_used >= 6) else dom
        traffic = (tj.get("two_pass", {}) if form_used == 3 else tj).get(tkey)
    stages = {}
    for k, ms in stage_ms.items():
        sec = ms / 1e3 / trials_prof
        stages[k] = {"us_per_trial": sec * 1e6, "kernel": stage_kernels[k],
                     "gbs": per_trial_bytes[k] / sec / 1e9 if sec > 0 else None}
    achieved = stages[dom]["gbs"]
    out = {"bound": "hbm", "kernel": stage_kernels[dom], "stage": dom, "achieved": achieved,
           "peak": peak, "unit": "GB/s", "frac": achieved / peak if achieved else None,
           "traffic": traffic, "peak_kind": peak_kind, "bytes_per_trial": per_trial_bytes[dom],
           "stages": stages}
    if dom == "harm":
        # the harmonic kernel's limiter is the SM's shared-memory bandwidth
        # (128 B per clock): per output bin 31 fraction loads + 1 tile load
        # (one 4-byte lane word each, 128 B) plus the windows the tensor
        # copies write (16.5 floats, 66 B)
        out["limiter"] = "shared-memory bandwidth (tensor-copy writes + 32 loads per bin)"
        out["smem_bytes_per_trial"] = 194.0 * B
        if sm_mhz:
            sec = stages["harm"]["us_per_trial"] / 1e6
            smem_peak = 128.0 * 148 * sm_mhz * 1e6
            out["smem_gbs"] = 194.0 * B / sec / 1e9
            out["smem_peak_gbs"] = smem_peak / 1e9
            out["smem_frac"] = 194.0 * B / sec / smem_peak
    return out


def _timed_block(eng, rows, dms, stream, chunk):
    """Searches rows in chunks through psx_search_block; CUDA-event time on
    the engine's stream.  Returns (seconds, candidate arrays per chunk)."""
    import torch
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    outs = []
    for c0 in range(0, len(rows), chunk):
        idx = np.arange(c0, min(len(rows), c0 + chunk))
        outs.append(eng.search_block([rows[i] for i in idx], dms[idx], idx.astype(np.int32))[0])
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3, outs


def run_config3(args, emit=True):
    """2048 DM trials x 2^22 samples of the small benchmark's statistics,
    acc +-50, 4 folds, S/N 7: batched (autotuned) over every DM trial, plain
    on a sample, and the candidate sets of the sampled DM trials compared."""
    import torch
    from peasoup_b200 import search, synth
    from peasoup_b200.build import build
    from peasoup_b200.transforms import AccelerationPlan
    build()
    n, ts, ndm = 1 << 22, 64e-6, args.ndm or 2048
    t0 = time.perf_counter()
    block = _pulse_block_torch(ndm, n, ts, seed=3)
    torch.cuda.synchronize()
    log(f"config 3: synthesised {ndm} series in {time.perf_counter() - t0:.1f}s")
    dms = (0.5 * np.arange(ndm)).astype(np.float32)

    def params(mode, batch=0, shape=0):
        return search.SearchParams(fft_size=n, tsamp=ts, acc_lo=-50.0, acc_hi=50.0,
                                   nharmonics=4, min_snr=7.0, cfreq_hz=synth.CFREQ_HZ,
                                   ch_bw_hz=synth.CH_BW_HZ, mode=mode, batch=batch,
                                   harm_shape=shape, group_dms=args.group_dms)
    if args.batch:
        tune = {"batch": args.batch, "harm_shape": args.harm_shape}
    else:
        tune = search.autotune(params("batched"), batches=(4, 8, 16, 32), reps=4)
    ap = AccelerationPlan(-50.0, 50.0, 1.10, 64e-6, n, ts, synth.CFREQ_HZ, synth.CH_BW_HZ)
    ntr = [len(ap.generate_accel_list(float(d), 0.0)) for d in dms]
    stream = torch.cuda.Stream()
    eng = search.AccelSearch(params("batched", tune["batch"], tune["harm_shape"]))
    eng.set_stream(stream.cuda_stream)
    rows = [block[i] for i in range(ndm)]
    _timed_block(eng, rows[:16], dms[:16], stream, 16)          # warm-up
    eng.profile(reset=True)
    with ClockSampler(0) as clk:
        tb, outs_b = _timed_block(eng, rows, dms, stream, 64)
    clocks = clk.summary()
    hostp = eng.profile(reset=True)   # host times of the timed pass (no events)
    host_us = {k: 1e3 * hostp[k] / ndm for k in ("host_enqueue_ms", "host_wait_ms",
                                                  "host_collect_ms")}
    # per-stage device times (CUDA events around every launch group, no
    # graph capture) on the first 128 DM trials, for the stage roofline
    eng.set_profile(True)
    eng.profile(reset=True)
    _timed_block(eng, rows[:128], dms[:128], stream, 64)
    prof = eng.profile(reset=True)
    eng.set_profile(False)
    info = eng.info()
    peak, peak_kind = peaks()
    roofline = stage_roofline(prof, n, info["fft_form"], info["harm_shape"], peak, peak_kind,
                              sm_mhz=clocks.get("sm_mhz"))
    roofline["prologue_span_us_per_dm"] = 1e3 * prof["prologue_ms"] / max(1, prof["dms"])
    nsample = min(ndm, args.plain_sample)
    sel = np.linspace(0, ndm - 1, nsample).astype(int)
    engp = search.AccelSearch(params("plain"))
    engp.set_stream(stream.cuda_stream)
    _timed_block(engp, [rows[i] for i in sel[:2]], dms[sel[:2]], stream, 2)
    tp, outs_p = _timed_block(engp, [rows[i] for i in sel], dms[sel], stream, 64)
    # candidate sets of the sampled DM trials: plain vs batched
    cb = np.concatenate(outs_b)
    cp = np.concatenate(outs_p)
    bsel = cb[np.isin(cb["dm_idx"], sel)]
    cp_fixed = cp.copy()
    cp_fixed["dm_idx"] = sel[cp["dm_idx"]]          # plain ran on a subset: map back
    cp_fixed["dm"] = dms[cp_fixed["dm_idx"]]
    key = lambda c: (int(c["dm_idx"]), float(c["acc"]), int(c["nh"]), float(c["freq"]))
    kb = {key(c): float(c["snr"]) for c in bsel}
    kp = {key(c): float(c["snr"]) for c in cp_fixed}
    same = set(kb) == set(kp)
    worst = max([abs(kb[k] - kp[k]) / max(abs(kp[k]), 1e-30) for k in set(kb) & set(kp)] or [0])
    tot_b = sum(ntr)
    tot_p = sum(ntr[i] for i in sel)
    vb, vp = tot_b / tb, tot_p / tp
    eng.close()
    engp.close()
    line = {
        "metric": "DM x accel trials/s, config 3 (2048 DM x 2^22)", "config_id": 3,
        "value": vb, "unit": "trials/s", "higher_is_better": True,
        "batched": {"value": vb, "seconds": tb, "dm_trials": ndm, "trials": tot_b,
                    "batch": tune["batch"], "harm_shape": tune["harm_shape"],
                    "group_dms": info["group_dms"]},
        "plain": {"value": vp, "seconds": tp, "dm_trials": int(nsample), "trials": tot_p},
        "batched_over_plain": vb / vp,
        "candidate_sets_equal_on_plain_sample": bool(same),
        "candidates_compared": len(kp), "snr_worst_rel": worst,
        "hbm_roofline_frac": (ndm * 24.0 * n + tot_b * 12.0 * n) / tb / (peaks()[0] * 1e9),
        "roofline": roofline,
        "host_us_per_dm": host_us,
        "clocks": clocks,
        "workload": "2048 DM x 2^22, tsamp 64us, white N(0,1) + P=5.7ms 5% duty 0.3 sigma "
                    "pulsar at +12 m/s^2 in every row, acc -50..50 (15 trials at DM 0), "
                    "4 folds, S/N 7, no zap list; series resident on the GPU",
    }
    del block, rows
    torch.cuda.empty_cache()
    if emit:
        print(json.dumps(line), flush=True)
    return line



def run_config5(args, emit=True):
    """2^27 samples, 64 DM trials, acc +-500 (123,653 trials at DM 0), 5
    folds: a fixed subset timed and extrapolated.  Per-trial and per-DM
    costs come from two subsets of different trial counts on the same DM
    trials (narrowed acceleration ranges; the cost of a trial does not depend
    on its acceleration)."""
    import torch
    from peasoup_b200 import search, synth
    from peasoup_b200.build import build
    from peasoup_b200.transforms import AccelerationPlan
    build()
    n, ts, ndm = 1 << 27, 64e-6, 64
    nuse = args.ndm or 4
    plan = synth.survey_plan(ndm=ndm, nsamps=n, tsamp=ts, seed=5, npulsars=3, nbirdies=0)
    rng = np.random.default_rng(5)
    for p in plan.pulsars:
        p.accel = float(rng.uniform(-400.0, 400.0))
    dsel = list(range(nuse))
    t0 = time.perf_counter()
    block = synth.survey_block_torch(plan, dm_indices=dsel, chunk=1)
    torch.cuda.synchronize()
    log(f"config 5: synthesised {nuse} series of 2^27 in {time.perf_counter() - t0:.1f}s")
    ap = AccelerationPlan(-500.0, 500.0, 1.10, 64e-6, n, ts, synth.CFREQ_HZ, synth.CH_BW_HZ)
    full = [len(ap.generate_accel_list(float(d), 0.0)) for d in plan.dms]

    def params(mode, half, batch=0, shape=0):
        return search.SearchParams(fft_size=n, tsamp=ts, acc_lo=-half, acc_hi=half,
                                   nharmonics=5, min_snr=9.0, cfreq_hz=synth.CFREQ_HZ,
                                   ch_bw_hz=synth.CH_BW_HZ, mode=mode, batch=batch,
                                   harm_shape=shape)

    def ntrials(half, dlist):
        a = AccelerationPlan(-half, half, 1.10, 64e-6, n, ts, synth.CFREQ_HZ, synth.CH_BW_HZ)
        return sum(len(a.generate_accel_list(float(plan.dms[d]), 0.0)) for d in dlist)

    tune = search.autotune(params("batched", 500.0), batches=(2, 4, 8), reps=1,
                           max_trials=64)
    stream = torch.cuda.Stream()
    rows = [block[i] for i in range(nuse)]
    res = {}
    for mode, halves in (("batched", (0.5, 2.0)), ("plain", (0.25, 1.0))):
        fit = []
        for half in halves:
            eng = search.AccelSearch(params(mode, half, tune["batch"] if mode == "batched" else 0,
                                            tune["harm_shape"]))
            eng.set_stream(stream.cuda_stream)
            _timed_block(eng, rows[:1], plan.dms[:1], stream, 1)   # warm-up
            sec, _ = _timed_block(eng, rows, plan.dms[dsel], stream, nuse)
            fit.append((ntrials(half, dsel), sec))
            eng.close()
        (n1, s1), (n2, s2) = fit
        per_trial = (s2 - s1) / (n2 - n1)
        per_dm = max(0.0, (s1 - n1 * per_trial) / nuse)
        tot = sum(full)
        est = ndm * per_dm + tot * per_trial
        res[mode] = {"value": tot / est, "per_trial_us": 1e6 * per_trial,
                     "per_dm_ms": 1e3 * per_dm, "subset": [{"trials": a, "seconds": b}
                                                           for a, b in fit]}
    # per-stage device times of the batched engine (CUDA events around every
    # launch group) on the larger subset, for the roofline of its stages
    eng = search.AccelSearch(params("batched", 2.0, tune["batch"], tune["harm_shape"]))
    eng.set_stream(stream.cuda_stream)
    eng.set_profile(True)
    _timed_block(eng, rows, plan.dms[dsel], stream, nuse)
    prof = eng.profile(reset=True)
    info = eng.info()
    eng.close()
    peak, peak_kind = peaks()
    roofline = stage_roofline(prof, n, info["fft_form"], info["harm_shape"], peak, peak_kind)
    line = {
        "metric": "DM x accel trials/s, config 5 (2^27, 64 DM, acc +-500), extrapolated",
        "config_id": 5, "value": res["batched"]["value"], "unit": "trials/s",
        "higher_is_better": True, "batched": res["batched"], "plain": res["plain"],
        "batched_over_plain": res["batched"]["value"] / res["plain"]["value"],
        "trials_full": int(sum(full)), "trials_dm0": full[0],
        "batch": tune["batch"], "harm_shape": tune["harm_shape"],
        "fft_form": FFT_FORMS.get(info["fft_form"], str(info["fft_form"])),
        "roofline": roofline,
        "hbm_roofline_frac": ((24.0 * n * ndm + 12.0 * n * sum(full)) /
                              (ndm * res["batched"]["per_dm_ms"] / 1e3 +
                               sum(full) * res["batched"]["per_trial_us"] / 1e6) /
                              (peaks()[0] * 1e9)),
        "workload": f"2^27 x tsamp 64us, survey-shape red noise + 3 binary pulsars "
                    f"(|a| <= 400), 64 DM trials (0.5 steps), acc -500..500, 5 folds, S/N 9; "
                    f"timed on {nuse} DM trials with narrowed acceleration ranges "
                    f"(batched +-0.5 and +-2, plain +-0.25 and +-1 m/s^2) and extrapolated "
                    f"to the full {sum(full)} trials",
    }
    del block, rows
    torch.cuda.empty_cache()
    if emit:
        print(json.dumps(line), flush=True)
    return line


# ----------------------------------------------------------------- main arm
def run_psx(args, ws, rank, local):
    import torch
    from peasoup_b200 import search, synth
    from peasoup_b200.build import build
    build()
    peak, peak_kind = peaks()
    S = args.dms_per_step
    plan = synth.survey_plan(ndm=NDM, nsamps=N_FFT, tsamp=TSAMP)
    warm = dm_schedule(rank, ws, args.warmup, S, offset=args.steps)
    timed = dm_schedule(rank, ws, args.steps, S)
    need = sorted({d for st in warm + timed for d in st})
    t0 = time.perf_counter()
    block = synth.survey_block_torch(plan, dm_indices=need)
    torch.cuda.synchronize()
    row = {d: i for i, d in enumerate(need)}
    log(f"[rank {rank}] synthesised {len(need)} series in {time.perf_counter() - t0:.1f}s")

    # ---- autotuner (untimed): trials per launch group x harmonic-kernel shape
    tune = None
    batch, shape = args.batch, args.harm_shape
    if not args.batch:
        t0 = time.perf_counter()
        tune = search.autotune(make_params(plan, "batched"), batches=(16, 32, 48, 63, 64, 96, 128),
                               reps=2)
        batch, shape = tune["batch"], tune["harm_shape"]
        log(f"[rank {rank}] autotune: batch {batch}, harmonic shape {shape} "
            f"({time.perf_counter() - t0:.1f}s)")
    stream = torch.cuda.Stream()
    pr = make_params(plan, "batched", batch, shape)
    pr.graph = not args.no_graph
    pr.lanes = args.lanes
    pr.fft_form = args.fft_form
    eng = search.AccelSearch(pr)
    eng.set_stream(stream.cuda_stream)

    def do_step(dm_list, src):
        rows = [src[row[d]] for d in dm_list] if src is block else [src[d] for d in dm_list]
        return eng.search_block(rows, plan.dms[dm_list], np.array(dm_list, np.int32))

    # ---- warm-up (untimed)
    for st in warm:
        do_step(st, block)
    torch.cuda.synchronize()

    # ---- timed: series resident in HBM (graph-captured trial schedules)
    ntr = sum(trials_of(plan, st) for st in timed)
    launches = 0
    ncand = 0
    eng.profile(reset=True)
    with ClockSampler(local) as clk:
        barrier(ws)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for st in timed:
            c = do_step(st, block)[0]
            ncand += len(c)
            launches += eng.info()["kernel_launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
    dt = e0.elapsed_time(e1) / 1e3
    hostp = eng.profile(reset=True)   # host times of the timed steps (no events)
    ndm_timed = max(1, sum(len(st) for st in timed))
    host_us = {k: 1e3 * hostp[k] / ndm_timed for k in ("host_enqueue_ms", "host_wait_ms",
                                                        "host_collect_ms")}
    batch_used = eng.info()["batch"]
    shape_used = eng.info()["harm_shape"]
    form_used = eng.info()["fft_form"]
    dt_max = max_over_ranks(ws, dt)
    tot_trials = sum_over_ranks(ws, ntr)
    value = tot_trials / dt_max
    clocks = clk.summary()

    # ---- the same steps again with CUDA events around every launch group
    # on the engine's stream (per-stage device time; graph capture is off
    # while events are recorded)
    eng.set_profile(True)
    eng.profile(reset=True)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for st in timed:
        do_step(st, block)
    p1.record(stream)
    torch.cuda.synchronize()
    prof = eng.profile(reset=True)
    eng.set_profile(False)
    value_profiled = tot_trials / max_over_ranks(ws, p0.elapsed_time(p1) / 1e3)

    # ---- e2e through the C ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        host = {}
        for st in timed + warm[:1]:
            for d in st:
                if d not in host:
                    h = torch.empty(N_FFT, dtype=torch.float32, pin_memory=True)
                    h.copy_(block[row[d]])
                    host[d] = h.numpy()
        do_step(warm[0] if warm else timed[0], host)
        torch.cuda.synchronize()
        barrier(ws)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        nc2 = 0
        for st in timed:
            c = do_step(st, host)[0]
            nc2 += len(c)
        f1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        dte = max_over_ranks(ws, f0.elapsed_time(f1) / 1e3)
        e2e = {"value": tot_trials / dte, "unit": "trials/s",
               "h2d_bytes_per_step": S * N_FFT * 4,
               "d2h_bytes_per_step": int(nc2 / max(1, len(timed))) * 24}
        del host

    # ---- plain path (one trial per launch) on a sample
    plain = None
    if not args.no_plain:
        eng_p = search.AccelSearch(make_params(plan, "plain"))
        eng_p.set_stream(stream.cuda_stream)
        ps = timed[:max(1, len(timed) // 4)]
        eng_p.search_block([block[row[d]] for d in ps[0][:1]], plan.dms[ps[0][:1]])
        torch.cuda.synchronize()
        barrier(ws)
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for st in ps:
            eng_p.search_block([block[row[d]] for d in st], plan.dms[st])
        g1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        dtp = max_over_ranks(ws, g0.elapsed_time(g1) / 1e3)
        ntp = sum_over_ranks(ws, sum(trials_of(plan, st) for st in ps))
        plain = {"value": ntp / dtp, "unit": "trials/s", "steps": len(ps),
                 "batched_over_plain": value / (ntp / dtp)}
        eng_p.close()

    # ---- roofline of the dominant stage (CUDA events on the engine stream)
    roofline = stage_roofline(prof, N_FFT, form_used, shape_used, peak, peak_kind,
                              sm_mhz=clocks.get("sm_mhz"))
    roofline.update({
        "prologue_span_us_per_dm": 1e3 * prof["prologue_ms"] / max(1, prof["dms"]),
        "prologue_note": "the prologue of DM d+1 runs on its own stream alongside the "
                         "trials of DM d, so its span includes sharing the GPU",
        "timing": "CUDA events per launch group on the engine stream, over a "
                  "re-run of the timed steps without graph capture "
                  f"({value_profiled:.0f} trials/s)"})
    # end-to-end algorithmic roofline of the whole search (12N per trial,
    # 24N per DM prologue)
    ndm_total = sum_over_ranks(ws, sum(len(st) for st in timed))
    alg = (ndm_total * 24.0 * N_FFT + tot_trials * 12.0 * N_FFT) / dt_max
    hbm_frac = alg / (peak * 1e9)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        d0 = timed[0][0]
        x = block[row[d0]].cpu().numpy()
        cpu_v, threads, cpu_tr, cpu_s = cpu_baseline(plan, x, plan.dms[d0])
        cpu = {"value": cpu_v, "unit": "trials/s", "cores": threads, "kind": "port",
               "sample": (f"FP32 C++ rendering of the same stages (oracle/cpu_render.cpp; "
                          f"libtorch's MKL FFT in place of FFTW, absent in the image) on one "
                          f"whole DM trial of the workload (DM {float(plan.dms[d0]):g}, "
                          f"{cpu_tr} acceleration trials) on {threads} host threads: "
                          f"{cpu_s:.2f}s; the FP64 oracle is the checker only")}
    eng.close()
    served = None
    block = None   # the survey block is not needed any more
    torch.cuda.empty_cache()
    if rank == 0 and ws == 1 and args.served > 0:
        t0 = time.perf_counter()
        served = run_served(args.served, rank, "served", args.served_policy,
                            args.served_slots)
        log(f"[rank {rank}] served workload in {time.perf_counter() - t0:.1f}s")
    other_configs = None
    if rank == 0 and ws == 1 and not args.no_configs:
        # the batched form at scale (config 3) and the long segment (config
        # 5), each with its plain comparison and stage roofline
        import argparse as _ap
        t0 = time.perf_counter()
        sub = _ap.Namespace(**vars(args))
        sub.ndm = 0
        sub.batch, sub.harm_shape = 0, 0   # each config tunes its own
        other_configs = {"3": run_config3(sub, emit=False), "5": run_config5(sub, emit=False)}
        log(f"[rank {rank}] configs 3 and 5 in {time.perf_counter() - t0:.1f}s")
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "trials/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt_max / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded survey-shape series made on the GPU)",
            "config": {"workload": "survey-2^23: 256 DM trials x 2^23 samples, tsamp 76us, "
                                   "acc -100..100, 5 folds, S/N 9, 20 birdies zapped",
                       "dms_per_step": S, "mode": "batched",
                       "batch": batch_used, "harm_shape": shape_used,
                       "graphs": not args.no_graph, "lanes": args.lanes or 1,
                       "fft_form": FFT_FORMS.get(form_used, str(form_used)),
                       "tuned": "autotuner (batch x harmonic shape)" if tune else "fixed",
                       "parallelism": f"dm-sharded x{ws}",
                       "l2": "inputs larger than L2 (8 x 32 MB series per step)"},
            "hbm_roofline_frac": hbm_frac,
            "plain": plain, "e2e": e2e, "served": served, "roofline": roofline,
            "other_configs": other_configs,
            "cpu_baseline": cpu,
            "host_us_per_dm": host_us,
            "clocks": clocks, "gpu_launches": launches, "candidates": ncand,
            "trials": int(tot_trials),
        }
        print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------- profiling case
def run_case(args):
    """A small search case for profiler captures (not a benchmark): the
    first --ndm (default 2) DM trials of the survey workload, searched one
    DM trial per call by the batched engine with CUDA events around every
    launch group (so no graph capture: each kernel is an ordinary stream
    launch), --batch / --harm-shape / --fft-form as given.  Two DM trials
    hold about 1.5 GB on the device, so a capture of any of its kernels
    stays small while every buffer a kernel streams exceeds the 126 MB L2.
    Prints one JSON line with the engine's counters and stage times."""
    import torch
    from peasoup_b200 import search, synth
    from peasoup_b200.build import build
    build()
    ndm = args.ndm or 2
    n = args.case_nsamps or N_FFT
    plan = synth.survey_plan(ndm=NDM, nsamps=n, tsamp=TSAMP)
    block = synth.survey_block_torch(plan, dm_indices=list(range(ndm)))
    pr = make_params(plan, "batched", args.batch, args.harm_shape)
    pr.fft_size = n
    pr.fft_form = args.fft_form
    if args.case_acc > 0:
        pr.acc_lo, pr.acc_hi = -args.case_acc, args.case_acc
    s = search.AccelSearch(pr)
    s.set_profile(True)
    counts = []
    for d in range(ndm):
        counts.append(len(s.search(block[d], float(plan.dms[d]), d)[0]))
    torch.cuda.synchronize()
    print(json.dumps({"workload": "case", "nsamps": n, "ndm": ndm, "candidates": counts,
                      "info": s.info(),
                      "profile": s.profile()}), flush=True)
    s.close()
    return 0


# ----------------------------------------------------------- dedispersion
DD_NCHANS = 64
DD_NBITS = 8


def _dd_job(job):
    """Oracle dedispersion of one sample (spawned worker); its elapsed time."""
    rows, nbits, nchans, delays, dms = job
    from oracle import oracle as O
    t0 = time.perf_counter()
    O.dedisperse(rows, nbits, nchans, delays, dms)
    return time.perf_counter() - t0


def run_dedisp(args, ws, rank, local):
    """The producer of the search's input: 2^23 samples x 64 channels of
    8-bit SIGPROC rows (tsamp 76 us, fch1 1510 MHz, foff -1.09 MHz)
    dedispersed to 256 DM trials (DM_i = 0.5 i) per step; each rank
    dedisperses its own block (weak scaling).  value = dedispersed samples
    per second with the rows resident in HBM; e2e = the same from pinned
    host rows through psx_dedisp_execute_host with one row of the result
    read back."""
    import ctypes as C
    import torch
    from peasoup_b200 import _lib, synth
    from peasoup_b200.build import build
    if rank == 0:
        build()
    barrier(ws)
    L = _lib.load()
    n = args.case_nsamps or N_FFT
    nchans = args.dd_nchans or DD_NCHANS
    nbits = args.dd_nbits or DD_NBITS
    ndm = args.ndm or NDM
    dms = (0.5 * np.arange(ndm)).astype(np.float32)
    plan = C.c_void_p()
    # the 64-channel band (1510 MHz down by 64 x 1.09 MHz) split into nchans
    foff = synth.FOFF_MHZ * DD_NCHANS / nchans
    _lib.check(L.psx_dedisp_create(nchans, TSAMP, synth.FCH1_MHZ, foff, C.byref(plan)),
               "dedisp_create")
    _lib.check(L.psx_dedisp_set_dm_list(plan, dms.ctypes.data, ndm), "set_dm_list")
    md = int(L.psx_dedisp_get_max_delay(plan))
    nout = n - md
    pitch = (nout + 3) // 4 * 4
    g = torch.Generator(device="cuda").manual_seed(7 + rank)
    rows = torch.randint(0, 256, (n, nchans * nbits // 8), dtype=torch.uint8, device="cuda",
                         generator=g)
    out = torch.empty((ndm, pitch), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    sh = C.c_void_p(stream.cuda_stream)

    def step_dev():
        _lib.check(L.psx_dedisp_execute(plan, n, C.c_void_p(rows.data_ptr()), nbits,
                                        C.c_void_p(out.data_ptr()), pitch, 0, sh), "execute")

    host = torch.empty(rows.shape, dtype=torch.uint8, pin_memory=True)
    host.copy_(rows)
    back = torch.empty(4096, dtype=torch.float32, pin_memory=True)

    def step_host():
        _lib.check(L.psx_dedisp_execute_host(plan, n, C.c_void_p(host.data_ptr()), nbits,
                                             C.c_void_p(out.data_ptr()), pitch, 0, sh),
                   "execute_host")
        with torch.cuda.stream(stream):
            back.copy_(out[ndm - 1, :4096], non_blocking=True)

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        stream.synchronize()
        barrier(ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        barrier(ws)
        return max_over_ranks(ws, e0.elapsed_time(e1) / 1e3)

    with ClockSampler(local) as clk:
        t_dev = timed(step_dev, args.steps, args.warmup)
    clocks = clk.summary()
    k_e2e = max(2, args.steps // 2)
    t_e2e = None if args.no_e2e else timed(step_host, k_e2e, 2)
    per = ndm * nout
    value = ws * per * args.steps / t_dev
    e2e = ws * per * k_e2e / t_e2e if t_e2e else None
    ms = t_dev / args.steps * 1e3
    alg = n * nchans * nbits / 8 + 2.0 * n * nchans + 4.0 * per
    peak, kind = peaks()
    achieved = alg / (t_dev / args.steps) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get("dedisp", {}).get("step_bytes")
    cpu = None
    if rank == 0 and not args.no_cpu:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        from oracle import oracle as O
        delays = O.delay_table(nchans, TSAMP, synth.FCH1_MHZ, foff)
        ns = (1 << 18) + md
        sample = rows[:ns].cpu().numpy()
        cores = _cpu_workers()
        sub = 8
        jobs = [(sample, nbits, nchans, delays, dms[i * sub:(i + 1) * sub])
                for i in range(min(cores, ndm // sub))]
        t0 = time.perf_counter()
        with ProcessPoolExecutor(len(jobs), mp_context=mp.get_context("spawn")) as ex:
            list(ex.map(_dd_job, jobs))
        tc = time.perf_counter() - t0
        cpu = {"value": len(jobs) * sub * (ns - md) / tc, "unit": "samples/s",
               "cores": len(jobs), "kind": "port",
               "sample": f"{len(jobs)} x {sub} DM trials x {ns - md} samples of the same rows, "
                         f"one spawned process per core, {tc:.1f} s wall"}
    L.psx_dedisp_destroy(plan)
    if rank == 0:
        print(json.dumps({
            "metric": f"dedispersed samples/s ({ndm} DM x 2^{n.bit_length() - 1}, {nchans} ch, "
                      f"{nbits}-bit)",
            "value": value, "unit": "samples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8->u32 sums->f32",
            "data": "synthetic (uniform random 8-bit rows, seeded)",
            "config": {"workload": f"dedisperse {n} samples x {nchans}-channel {nbits}-bit rows "
                                   f"(tsamp 76 us, 1510 MHz, {foff:.4g} MHz) to {ndm} DM "
                                   f"trials DM_i = 0.5 i",
                       "rows_mb": n * nchans / 1e6, "output_gb": 4.0 * per / 1e9,
                       "max_delay": md,
                       "l2": f"input {n * nchans * nbits / 8e6:.0f} MB, output "
                             f"{4.0 * per / 1e9:.2f} GB"},
            "e2e": None if e2e is None else {
                "value": e2e, "unit": "samples/s",
                "h2d_bytes_per_step": n * nchans * nbits // 8, "d2h_bytes_per_step": 16384},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "note": f"unpack + dedisperse per launch pair, {alg / 1e9:.2f} GB "
                                 f"algorithmic (packed rows read, channel-major samples "
                                 f"written and read once, series written); traffic from "
                                 f"one ncu capture of 32 DM trials, writes scaled to 256; "
                                 f"peak {kind}; the kernel is bound by integer issue, "
                                 f"not by HBM"},
            "cpu_baseline": cpu, "gpu_launches": 2 * args.steps, "clocks": clocks,
        }), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=32)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="psx", choices=["psx", "reference"])
    ap.add_argument("--dms-per-step", type=int, default=8)
    ap.add_argument("--batch", type=int, default=0,
                    help="trials per launch group (0: autotuned together with the shape)")
    ap.add_argument("--harm-shape", type=int, default=0,
                    help="with --batch: harmonic-kernel shape (0: the default shape)")
    ap.add_argument("--dd-nchans", type=int, default=0,
                    help="--workload dedisp: channels (default 64)")
    ap.add_argument("--dd-nbits", type=int, default=0,
                    help="--workload dedisp: bits per sample (default 8)")
    ap.add_argument("--group-dms", type=int, default=0,
                    help="DM trials per grouped prologue (0: default rule, 1: off)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip configs 3 and 5 in the default run")
    ap.add_argument("--fft-form", type=int, default=0,
                    help="0: default (3 where the length allows it); 1: cuFFT complex "
                         "transform + fused unpack/interbin/normalise; 2: the reference's "
                         "real transform + interbin/normalise; 3: the library's two-pass "
                         "transform with the resample gather in its first pass")
    ap.add_argument("--lanes", type=int, default=0,
                    help="streams the launch groups alternate over (0: the engine's default)")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch the trial schedules directly instead of as CUDA graphs")
    ap.add_argument("--served", type=int, default=SERVED_REQUESTS,
                    help="requests of the served workload (0: skip)")
    ap.add_argument("--served-slots", type=int, default=SERVED_SLOTS,
                    help="served workload: requests admitted at once by the sharing policies")
    ap.add_argument("--served-policy", default="exclusive",
                    choices=["least_work", "even", "exclusive"],
                    help="scheduling between running requests of the served workload")
    ap.add_argument("--config", type=int, default=2, choices=[2, 3, 5],
                    help="2: the headline survey workload; 3 and 5: the other throughput "
                         "configurations (one JSON line each)")
    ap.add_argument("--case-nsamps", type=int, default=0,
                    help="--workload case / dedisp: samples (default 2^23)")
    ap.add_argument("--case-acc", type=float, default=0.0,
                    help="--workload case: acceleration half-range (default 100 m/s^2)")
    ap.add_argument("--ndm", type=int, default=0,
                    help="configs 3/5: DM trials to time; --workload case: DM trials "
                         "searched; --workload dedisp: DM trials (default 256)")
    ap.add_argument("--plain-sample", type=int, default=128,
                    help="config 3: DM trials searched by the plain path")
    ap.add_argument("--workload", default="search", choices=["search", "dedisp", "case"],
                    help="dedisp: the dedispersion producer instead of the search; case: a "
                         "small search case for profiler captures (--ndm DM trials, default 2)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    ws, rank, local = dist_init()
    try:
        if args.workload == "case":
            rc = run_case(args)
        elif args.workload == "dedisp":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable": (
                        "the reference dedisperses through the external dedisp library, "
                        "which is neither in the reference tree nor in this image")}))
                rc = 0
            else:
                rc = run_dedisp(args, ws, rank, local)
        elif args.impl == "reference":
            rc = run_reference(args, ws, rank)
        elif args.config == 3:
            run_config3(args)
            rc = 0
        elif args.config == 5:
            run_config5(args)
            rc = 0
        else:
            rc = run_psx(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
