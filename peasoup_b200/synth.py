"""Seeded synthetic dedispersed time series for the search workloads.

No survey data is available offline, so every workload is synthetic:
white noise, optional 1/f^1.5 red noise below 1 Hz, optional uint8
quantisation, injected accelerated pulsars and sinusoidal birdies.

A pulsar of spin frequency f0 and line-of-sight acceleration a is injected
with pulse phase phi(n) = f0*tsamp*(n - k*n*(n - N)), k = a*tsamp/(2c), the
sign convention of the reference's resampler (src/kernels.cu:321-324,
:361): resampleII(a) straightens it.  Pulses are Gaussian with FWHM =
duty*P.

Two backends: numpy (PCG64, used by tests and fixtures) and torch on the
GPU (used to make the large benchmark blocks quickly); they do not produce
identical numbers.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

C_LIGHT = 299792458.0

# Synthetic header: fch1 1510 MHz, foff -1.09 MHz, 64 channels (the values
# of the reference's example filterbank); centre frequency as the
# reference's SigprocFilterbank::get_cfreq computes it, in float.
FCH1_MHZ = 1510.0
FOFF_MHZ = -1.09
NCHANS = 64
CFREQ_MHZ = float(np.float32(FCH1_MHZ + FOFF_MHZ * NCHANS / 2))
CFREQ_HZ = float(np.float32(np.float64(np.float32(CFREQ_MHZ)) * 1e6))
CH_BW_HZ = float(np.float32(np.float64(np.float32(FOFF_MHZ)) * 1e6))


@dataclass
class Pulsar:
    period: float          # s
    accel: float           # m/s^2
    duty: float            # FWHM / period
    amp: float             # peak amplitude (absolute units)
    phase0: float = 0.0


@dataclass
class SeriesSpec:
    nsamps: int
    tsamp: float
    sigma: float = 1.0
    mean: float = 0.0
    red_noise: bool = False
    quantise_u8: bool = False
    pulsars: List[Pulsar] = field(default_factory=list)
    birdies: Optional[np.ndarray] = None   # frequencies (Hz) of injected sinusoids
    birdie_amp: float = 0.0


def pulse_train(n: int, tsamp: float, p: Pulsar, fft_size: Optional[int] = None) -> np.ndarray:
    N = fft_size or n
    k = p.accel * tsamp / (2.0 * C_LIGHT)
    i = np.arange(n, dtype=np.float64)
    phi = (i - k * i * (i - N)) * (tsamp / p.period) + p.phase0
    d = phi - np.round(phi)
    sig = p.duty / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    return p.amp * np.exp(-0.5 * (d / sig) ** 2)


def red_noise_np(rng: np.random.Generator, n: int, tsamp: float, sigma: float) -> np.ndarray:
    """1/f^1.5 noise below 1 Hz whose spectral level meets the white level
    (sigma^2 per sample) at 1 Hz."""
    nb = n // 2 + 1
    f = np.arange(nb) / (n * tsamp)
    srel = np.zeros(nb)
    m = (f > 0) & (f < 1.0)
    srel[m] = f[m] ** -1.5
    z = (rng.standard_normal(nb) + 1j * rng.standard_normal(nb)) / np.sqrt(2.0)
    Z = sigma * np.sqrt(n) * np.sqrt(srel) * z
    return np.fft.irfft(Z, n=n)


def make_series_np(spec: SeriesSpec, seed, fft_size: Optional[int] = None) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n = spec.nsamps
    x = spec.mean + spec.sigma * rng.standard_normal(n)
    if spec.red_noise:
        x += red_noise_np(rng, n, spec.tsamp, spec.sigma)
    for p in spec.pulsars:
        x += pulse_train(n, spec.tsamp, p, fft_size)
    if spec.birdies is not None and spec.birdie_amp:
        t = np.arange(n) * spec.tsamp
        for fb in spec.birdies:
            x += spec.birdie_amp * np.sin(2 * np.pi * fb * t + rng.uniform(0, 2 * np.pi))
    if spec.quantise_u8:
        x = np.clip(np.round(x), 0, 255)
    return x.astype(np.float32)


# ---------------------------------------------------------------- workloads
def config1_series(seed: int = 0, nsamps: int = 1 << 20, tsamp: float = 64e-6) -> np.ndarray:
    """White N(0,1) noise plus a P=5.7 ms, 5% duty, 0.3 sigma pulsar at
    +12 m/s^2."""
    spec = SeriesSpec(nsamps=nsamps, tsamp=tsamp, sigma=1.0,
                      pulsars=[Pulsar(period=5.7e-3, accel=12.0, duty=0.05, amp=0.3)])
    return make_series_np(spec, seed)


@dataclass
class SurveyBlock:
    """A block of DM trials at survey shape (the plain-method survey
    workload): uint8-quantised noise (mean 128, sigma 20) with 1/f^1.5 red
    noise, five pulsars at random DM indices, 20 birdies."""
    ndm: int
    nsamps: int
    tsamp: float
    dms: np.ndarray
    pulsar_dm_idx: np.ndarray
    pulsars: List[Pulsar]
    birdie_freqs: np.ndarray
    birdie_widths: np.ndarray

    def zaplist_text(self) -> str:
        return "".join(f"{f:.3f} {w:.3f}\n" for f, w in zip(self.birdie_freqs, self.birdie_widths))


def survey_plan(ndm: int = 256, nsamps: int = 1 << 23, tsamp: float = 76e-6, seed: int = 2,
                npulsars: int = 5, nbirdies: int = 20, dm_step: float = 0.5) -> SurveyBlock:
    rng = np.random.default_rng(seed)
    dms = (dm_step * np.arange(ndm)).astype(np.float32)
    pidx = rng.choice(ndm, size=min(npulsars, ndm), replace=False)
    pulsars = [Pulsar(period=float(np.exp(rng.uniform(np.log(2e-3), np.log(0.5)))),
                      accel=float(rng.uniform(-80, 80)), duty=float(rng.uniform(0.02, 0.10)),
                      amp=0.5 * 20.0, phase0=float(rng.uniform()))
               for _ in range(len(pidx))]
    bf = np.sort(rng.uniform(1.0, 1000.0, nbirdies)).astype(np.float32)
    bw = np.full(nbirdies, 0.1, np.float32)
    return SurveyBlock(ndm, nsamps, tsamp, dms, pidx, pulsars, bf, bw)


def survey_series_np(plan: SurveyBlock, dm_index: int, seed: int = 2) -> np.ndarray:
    ps = [plan.pulsars[j] for j in range(len(plan.pulsars)) if plan.pulsar_dm_idx[j] == dm_index]
    spec = SeriesSpec(nsamps=plan.nsamps, tsamp=plan.tsamp, sigma=20.0, mean=128.0,
                      red_noise=True, quantise_u8=True, pulsars=ps, birdies=plan.birdie_freqs,
                      birdie_amp=2.0)
    return make_series_np(spec, [seed, dm_index])


def survey_block_torch(plan: SurveyBlock, seed: int = 2, device: str = "cuda",
                       dm_indices=None, chunk: int = 8, out=None):
    """The survey block generated on the GPU with torch (fast at 2^23):
    returns a float32 tensor [len(dm_indices), nsamps].  Rows are made in
    chunks; the birdie sinusoids (common to every DM trial, as RFI is) are
    summed once."""
    import torch
    idx = list(range(plan.ndm)) if dm_indices is None else list(dm_indices)
    n, ts = plan.nsamps, plan.tsamp
    if out is None:
        out = torch.empty((len(idx), n), dtype=torch.float32, device=device)
    nb = n // 2 + 1
    f = torch.arange(nb, device=device, dtype=torch.float64) / (n * ts)
    srel = torch.zeros(nb, device=device, dtype=torch.float64)
    m = (f > 0) & (f < 1.0)
    srel[m] = f[m] ** -1.5
    amp_red = (20.0 * np.sqrt(n) / np.sqrt(2.0)) * torch.sqrt(srel)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed) * 7919 + 17)
    t = torch.arange(n, device=device, dtype=torch.float64) * ts
    ph = torch.rand(len(plan.birdie_freqs), generator=g, device=device,
                    dtype=torch.float64) * 2 * np.pi
    birdies = torch.zeros(n, device=device, dtype=torch.float64)
    for b, fb in enumerate(plan.birdie_freqs):
        birdies += 2.0 * torch.sin(2 * np.pi * float(fb) * t + ph[b])
    del t
    for c0 in range(0, len(idx), chunk):
        rows = idx[c0:c0 + chunk]
        g.manual_seed(int(seed) * 1000003 + int(rows[0]))
        x = 128.0 + 20.0 * torch.randn((len(rows), n), generator=g, device=device,
                                       dtype=torch.float64)
        z = torch.complex(torch.randn((len(rows), nb), generator=g, device=device,
                                      dtype=torch.float64),
                          torch.randn((len(rows), nb), generator=g, device=device,
                                      dtype=torch.float64))
        x += torch.fft.irfft(z * amp_red, n=n)
        del z
        x += birdies
        for r, d in enumerate(rows):
            for j, p in enumerate(plan.pulsars):
                if plan.pulsar_dm_idx[j] != d:
                    continue
                k = p.accel * ts / (2.0 * C_LIGHT)
                i = torch.arange(n, device=device, dtype=torch.float64)
                phi = (i - k * i * (i - n)) * (ts / p.period) + p.phase0
                dd = phi - torch.round(phi)
                sig = p.duty / (2.0 * np.sqrt(2.0 * np.log(2.0)))
                x[r] += p.amp * torch.exp(-0.5 * (dd / sig) ** 2)
        out[c0:c0 + len(rows)] = torch.clamp(torch.round(x), 0, 255).to(torch.float32)
        del x
    return out


# ------------------------------------------------------------ filterbanks
K_DM_S = 4.15e3  # s MHz^2 cm^3 / pc, the dispersion constant of the delay table


@dataclass
class FilterbankSpec:
    """A SIGPROC block: nchans channels from fch1 downwards in steps of
    |foff|, nbits-bit samples around mid-range, and pulsars dispersed at
    `dm` (the arrival at channel c is delayed by K/tsamp*(f_c^-2 -
    fch1^-2)*dm samples)."""
    nsamps: int
    tsamp: float = 320e-6
    nchans: int = NCHANS
    nbits: int = 8
    fch1: float = FCH1_MHZ
    foff: float = FOFF_MHZ
    dm: float = 0.0
    sigma: float = 0.0          # per-channel noise in sample units (0: a quarter range)
    pulsars: List[Pulsar] = field(default_factory=list)


def filterbank_values(spec: FilterbankSpec, seed: int = 0) -> np.ndarray:
    """(nsamps, nchans) unsigned samples, seeded (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    top = (1 << spec.nbits) - 1
    sigma = spec.sigma or max(0.5, (top + 1) / 6.0)
    mean = top / 2.0
    f = spec.fch1 + spec.foff * np.arange(spec.nchans)
    delay = K_DM_S * (f ** -2 - spec.fch1 ** -2) * spec.dm  # seconds
    out = np.empty((spec.nsamps, spec.nchans), np.uint32 if spec.nbits == 16 else np.uint8)
    i = np.arange(spec.nsamps, dtype=np.float64)
    for c in range(spec.nchans):
        x = rng.standard_normal(spec.nsamps)
        for p in spec.pulsars:
            phi = (i * spec.tsamp - delay[c]) / p.period + p.phase0
            d = phi - np.round(phi)
            s = p.duty / (2.0 * np.sqrt(2.0 * np.log(2.0)))
            x += p.amp * np.exp(-0.5 * (d / s) ** 2)
        out[:, c] = np.clip(np.round(mean + sigma * x), 0, top)
    return out
