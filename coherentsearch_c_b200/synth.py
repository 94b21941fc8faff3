"""Seeded synthetic workloads for the coherent harmonic-sum search.

There is no public dataset for this path: the reference validates against
private survey files (README.md:434-478).  These generators produce the
inputs the search workloads are specified on -- float32 time series of a given
length and sample time with Gaussian noise, optional power-law red noise and
von Mises pulse trains scaled to a requested folded S/N -- plus PRESTO-style
.inf/.dat files (the format src/fileio.c:38-72 and src/datpipe.c:336-397 read)
and 8-bit filterbank blocks for dedispersion.

Everything is seeded (numpy PCG64) so a (seed, index) pair always yields the
same bytes.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Pulsar:
    f0: float            # spin frequency, Hz
    duty: float          # FWHM duty cycle (fraction of a period)
    snr: float           # folded (matched-filter) S/N of the whole series
    phase0: float = 0.0


@dataclass
class SeriesSpec:
    N: int
    dt: float = 64e-6
    seed: int = 12345
    pulsars: list = field(default_factory=list)
    red_index: float | None = None   # power-law index of an added red-noise term
    red_amp: float = 0.0             # its rms relative to the white noise
    sigma: float = 1.0


def von_mises_kappa(duty: float) -> float:
    """Concentration giving a von Mises pulse of FWHM = duty (in turns)."""
    return math.log(2.0) / (1.0 - math.cos(math.pi * duty))


def pulse_train(N: int, dt: float, p: Pulsar) -> np.ndarray:
    t = np.arange(N, dtype=np.float64) * dt
    phase = (t * p.f0 + p.phase0) % 1.0
    kappa = von_mises_kappa(p.duty)
    s = np.exp(kappa * (np.cos(2.0 * np.pi * phase) - 1.0))
    s -= s.mean()
    # matched-filter S/N against unit white noise is amp * ||s||
    amp = p.snr / math.sqrt(float(np.dot(s, s)))
    return amp * s


def red_noise(N: int, index: float, rng: np.random.Generator) -> np.ndarray:
    nf = N // 2 + 1
    f = np.arange(nf, dtype=np.float64)
    f[0] = 1.0
    amp = f ** (index / 2.0)
    amp[0] = 0.0
    spec = (rng.standard_normal(nf) + 1j * rng.standard_normal(nf)) * amp
    x = np.fft.irfft(spec, n=N)
    sd = x.std()
    return x / sd if sd > 0 else x


def make_series(spec: SeriesSpec) -> np.ndarray:
    """Float32 time series: white noise (+ red noise) + pulse trains."""
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    x = rng.standard_normal(spec.N) * spec.sigma
    if spec.red_index is not None and spec.red_amp > 0:
        x += spec.red_amp * spec.sigma * red_noise(spec.N, spec.red_index, rng)
    for p in spec.pulsars:
        x += spec.sigma * pulse_train(spec.N, spec.dt, p)
    return x.astype(np.float32)


def write_inf(path: str, N: int, dt: float, name: str = "synthetic",
              dm: float = 0.0) -> None:
    """PRESTO-style .inf with the keys src/fileio.c:52-67 reads."""
    with open(path, "w") as f:
        f.write(f" Data file name without suffix          =  {name}\n")
        f.write(" Telescope used                         =  Synthetic\n")
        f.write(f" Object being observed                  =  {name}\n")
        f.write(" Epoch of observation (MJD)             =  60000.000000000000\n")
        f.write(f" Number of bins in the time series      =  {N}\n")
        f.write(f" Width of each time series bin (sec)    =  {dt!r}\n")
        f.write(f" Dispersion measure (cm-3 pc)           =  {dm!r}\n")


def write_dat(stem: str, x: np.ndarray, dt: float, dm: float = 0.0) -> str:
    """Write <stem>.dat (float32) and <stem>.inf; returns the .dat path."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    x.tofile(stem + ".dat")
    write_inf(stem + ".inf", x.size, dt, name=os.path.basename(stem), dm=dm)
    return stem + ".dat"


# ---------------------------------------------------------------------------
# The workloads the search is specified on
# ---------------------------------------------------------------------------
def config_small(seed: int = 12345) -> SeriesSpec:
    """N=2^20, dt=64 us, N(0,1) + von Mises pulsar f0=7.3 Hz, duty 5%, S/N~15."""
    return SeriesSpec(N=1 << 20, dt=64e-6, seed=seed,
                      pulsars=[Pulsar(7.3, 0.05, 15.0)])


def config_precision(seed: int = 12346, N: int = 1 << 23) -> SeriesSpec:
    """N=2^23: three pulsars (1.7, 29.4, 311 Hz; duty 2-10%; S/N 10-40) plus
    power-law red noise of index -2."""
    return SeriesSpec(N=N, dt=64e-6, seed=seed,
                      pulsars=[Pulsar(1.7, 0.10, 40.0, 0.1),
                               Pulsar(29.4, 0.05, 20.0, 0.4),
                               Pulsar(311.0, 0.02, 10.0, 0.7)],
                      red_index=-2.0, red_amp=0.5)


def config_dm_sweep(n_files: int = 256, seed: int = 12347,
                    lo: int = 1 << 21, hi: int = 1 << 23, quantum: int = 1024):
    """Uneven-length list: lengths log-uniform in [lo, hi] (rounded to a
    multiple of `quantum` so every length is even), one pulsar of f0=11.2 Hz
    whose S/N peaks at list index n/2 with a Gaussian fall-off of width 8."""
    rng = np.random.Generator(np.random.PCG64(seed))
    specs = []
    centre = n_files // 2
    for i in range(n_files):
        N = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        N = max(quantum, (N // quantum) * quantum)
        snr = 25.0 * math.exp(-0.5 * ((i - centre) / 8.0) ** 2)
        pulsars = [Pulsar(11.2, 0.05, snr, 0.3)] if snr > 0.5 else []
        specs.append(SeriesSpec(N=N, dt=64e-6, seed=seed * 1000 + i,
                                pulsars=pulsars))
    return specs


# ---------------------------------------------------------------------------
# Spectra without the reference pipeline (workload generation for timing)
# ---------------------------------------------------------------------------
def packed_spectrum(x: np.ndarray) -> np.ndarray:
    """PRESTO packing of the forward real FFT: complex64[N/2] with bin 0
    holding (DC, Nyquist), as realfft writes it (src/datpipe.c:101-138)."""
    X = np.fft.rfft(x.astype(np.float64))
    n2 = x.size // 2
    out = np.empty(n2, dtype=np.complex64)
    out[1:] = X[1:n2]
    out[0] = complex(X[0].real, X[n2].real)
    return out


def normalised_spectrum(x: np.ndarray, block: int = 100) -> np.ndarray:
    """Packed spectrum scaled to unit mean power by block medians of the
    power (median/ln2, the rednoise noise estimate), bin 0 set to (1, 0).
    A vectorised stand-in for rednoise used only to build timing inputs."""
    S = packed_spectrum(x)
    n = S.size
    p = (S.real.astype(np.float64) ** 2 + S.imag.astype(np.float64) ** 2)
    nb = (n - 1) // block
    scale = np.ones(n, dtype=np.float64)
    if nb > 0:
        med = np.median(p[1:1 + nb * block].reshape(nb, block), axis=1) / math.log(2.0)
        med[med <= 0] = 1.0
        scale[1:1 + nb * block] = np.repeat(1.0 / np.sqrt(med), block)
        scale[1 + nb * block:] = 1.0 / math.sqrt(med[-1])
    out = (S * scale).astype(np.complex64)
    out[0] = 1.0 + 0.0j
    return out


def amps_interleaved(S: np.ndarray) -> np.ndarray:
    """complex64[n] -> float32[2n] (re, im interleaved), the FFTFile.amps layout."""
    return np.ascontiguousarray(S, dtype=np.complex64).view(np.float32)


# ---------------------------------------------------------------------------
# 8-bit filterbank (raw-data front end)
# ---------------------------------------------------------------------------
@dataclass
class FilterbankSpec:
    """SIGPROC-style 8-bit filterbank: per-channel N(mean, sigma) clipped to
    0..255 plus a dispersed von Mises pulsar.  Channels are stored highest
    frequency first, as SIGPROC files with negative foff hold them."""
    nchan: int = 1024
    nspec: int = 1 << 22
    fctr: float = 1400.0          # MHz
    bw: float = 300.0             # MHz
    dt: float = 64e-6
    mean: float = 128.0
    sigma: float = 12.0
    dm: float = 56.8
    f0: float = 4.1
    duty: float = 0.04
    amp: float = 2.0              # pulse peak per channel, in units of sigma
    seed: int = 4

    @property
    def chanwid(self) -> float:
        return self.bw / self.nchan

    @property
    def lofreq(self) -> float:
        """Centre of the lowest channel (PRESTO's idata.freq,
        third_party/presto/src/sigproc_fb.c:435-441)."""
        return self.fctr + 0.5 * self.chanwid - 0.5 * self.bw


def config_filterbank(nspec: int = 1 << 22, seed: int = 4) -> FilterbankSpec:
    """1024 channels, 1400 MHz centre, 300 MHz, 64 us, DM 56.8 pulsar at
    4.1 Hz with a 4 % duty cycle."""
    return FilterbankSpec(nspec=nspec, seed=seed)


def make_filterbank(spec: FilterbankSpec, chunk: int = 1 << 14) -> np.ndarray:
    """[nspec][nchan] uint8, highest frequency first."""
    rng = np.random.default_rng(spec.seed)
    freqs = spec.lofreq + spec.chanwid * np.arange(spec.nchan)            # ascending
    delay = spec.dm / (0.000241 * freqs * freqs)                           # seconds
    kappa = von_mises_kappa(spec.duty)
    out = np.empty((spec.nspec, spec.nchan), np.uint8)
    for t0 in range(0, spec.nspec, chunk):
        n = min(chunk, spec.nspec - t0)
        t = (t0 + np.arange(n))[:, None] * spec.dt
        phase = (spec.f0 * (t - delay[None, :])) % 1.0
        pulse = np.exp(kappa * (np.cos(2.0 * np.pi * phase) - 1.0))
        x = spec.mean + spec.sigma * (rng.standard_normal((n, spec.nchan)) + spec.amp * pulse)
        np.clip(np.rint(x), 0, 255, out=x)
        out[t0:t0 + n] = x[:, ::-1].astype(np.uint8)
    return out


def write_filterbank(path: str, raw: np.ndarray, spec: FilterbankSpec,
                     source_name: str = "SYNTH", tstart: float = 60000.0) -> None:
    """An 8-bit SIGPROC filterbank file of raw ([nspec][nchan], highest
    frequency first) with the header keywords PRESTO reads
    (third_party/presto/src/sigproc_fb.c:240-345): fch1 the highest channel,
    foff = -chanwid."""
    import struct

    def s(x: str) -> bytes:
        b = x.encode()
        return struct.pack("<i", len(b)) + b

    hdr = (s("HEADER_START") + s("source_name") + s(source_name) +
           s("telescope_id") + struct.pack("<i", 0) + s("machine_id") + struct.pack("<i", 0) +
           s("data_type") + struct.pack("<i", 1) +
           s("fch1") + struct.pack("<d", spec.lofreq + (spec.nchan - 1) * spec.chanwid) +
           s("foff") + struct.pack("<d", -spec.chanwid) +
           s("nchans") + struct.pack("<i", spec.nchan) + s("nbits") + struct.pack("<i", 8) +
           s("tstart") + struct.pack("<d", tstart) + s("tsamp") + struct.pack("<d", spec.dt) +
           s("nifs") + struct.pack("<i", 1) + s("HEADER_END"))
    raw = np.ascontiguousarray(raw, dtype=np.uint8)
    if raw.ndim != 2 or raw.shape[1] != spec.nchan:
        raise ValueError("raw must be [nspec][nchan] uint8")
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(raw.tobytes())
