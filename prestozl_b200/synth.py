"""Seeded synthetic pulsar spectra in PRESTO's ``.fft``/``.inf`` format.

The reference ships no data for the jerk search, so every input used by the
tests and the benchmark is generated here from a fixed seed:

* a white Gaussian time series (mean 0, sd 1) of ``N`` samples,
* plus pulsars whose phase follows PRESTO's Fourier-domain convention
  (``src/responses.c:388-393``): with ``u = t / T`` in [0, 1] and average
  Fourier frequency ``r``, f-dot ``z`` and f-dot-dot ``w`` (all in bins),
  ``r0 = r - z/2 + w/12``, ``z0 = z - w/2`` and the phase in cycles is
  ``phi(u) = r0*u + z0*u**2/2 + w*u**3/6``.  Harmonic ``k`` has phase
  ``k*phi`` and amplitude ``a_k`` proportional to ``1/k``.
* ``snr`` fixes the amplitudes: the ideal normalised power summed over the
  harmonics of a pulsar (``sum_k a_k**2 * N / 4`` for unit-variance noise)
  equals ``snr**2``.

The spectrum is the real FFT with PRESTO's packing (``src/fastffts.c:163-237``
``realfft``): ``N/2`` complex64 bins, bin 0 holding the DC term in its real
part and the Nyquist term in its imaginary part; the forward sign is
``exp(-2*pi*i*j*k/N)`` (numpy's ``rfft``).
"""

from __future__ import annotations

import dataclasses
import os
from typing import List, Sequence

import numpy as np


@dataclasses.dataclass(frozen=True)
class Pulsar:
    f: float          # average spin frequency (Hz)
    z: float          # average Fourier f-dot (bins drifted over T)
    w: float          # Fourier f-dot-dot (change of z over T)
    snr: float        # sqrt of the ideal summed normalised power
    nharm: int = 1    # number of harmonics, amplitudes proportional to 1/k
    phase: float = 0.0


def timeseries(N: int, dt: float, pulsars: Sequence[Pulsar], seed: int,
               chunk: int = 1 << 22) -> np.ndarray:
    """Float32 time series: seeded N(0, 1) noise plus the given pulsars."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(N).astype(np.float64)
    T = N * dt
    for p in pulsars:
        r = p.f * T
        r0 = r - 0.5 * p.z + p.w / 12.0
        z0 = p.z - 0.5 * p.w
        k = np.arange(1, p.nharm + 1, dtype=np.float64)
        amps = 1.0 / k
        # sum_k a_k^2 N / 4 = snr^2
        scale = p.snr / np.sqrt(np.sum(amps ** 2) * N / 4.0)
        amps = amps * scale
        for lo in range(0, N, chunk):
            u = np.arange(lo, min(N, lo + chunk), dtype=np.float64) / N
            phi = u * (r0 + u * (0.5 * z0 + u * (p.w / 6.0)))
            for kk, a in zip(k, amps):
                cyc = kk * phi
                cyc -= np.floor(cyc)
                x[lo:lo + len(u)] += a * np.cos(2.0 * np.pi * cyc + p.phase)
    return x.astype(np.float32)


def presto_fft(ts: np.ndarray) -> np.ndarray:
    """PRESTO-packed real FFT (complex64, N/2 bins) of an even-length series."""
    N = len(ts)
    if N % 2:
        raise ValueError("time series length must be even")
    X = np.fft.rfft(ts.astype(np.float64))
    out = X[: N // 2].astype(np.complex64)
    out[0] = np.complex64(complex(X[0].real, X[N // 2].real))
    return out


def write_inf(root: str, N: int, dt: float, note: str = "seeded synthetic") -> None:
    """Write a makedata-style ``.inf`` (``src/ioinf.c:121-240`` ``readinf``):
    'None (Artificial Data Set)' telescope, so no sky/band fields follow."""
    def line(key: str, val) -> str:
        return " " + key.ljust(39) + "=  " + str(val) + "\n"

    with open(root + ".inf", "w") as f:
        f.write(line("Data file name without suffix", os.path.basename(root)))
        f.write(line("Telescope used", "None (Artificial Data Set)"))
        f.write(line("Number of bins in the time series", N))
        f.write(line("Width of each time series bin (sec)", repr(float(dt))))
        f.write(line("Any breaks in the data? (1=yes, 0=no)", 0))
        f.write(line("Data analyzed by", "prestozl_b200.synth"))
        f.write(" Any additional notes:\n")
        f.write("    " + note + "\n")


def write_fft(root: str, spec: np.ndarray, N: int, dt: float) -> None:
    np.ascontiguousarray(spec, dtype=np.complex64).tofile(root + ".fft")
    write_inf(root, N, dt)


def read_fft(path: str) -> np.ndarray:
    return np.fromfile(path, dtype=np.complex64)


# --------------------------------------------------------------------------
# The named workloads.

def small_pulsar() -> List[Pulsar]:
    """One binary pulsar: f=123.4 Hz, 5 harmonics (1/k), z=+12, w=+40, SNR 15."""
    return [Pulsar(f=123.4, z=12.0, w=40.0, snr=15.0, nharm=5)]


def random_pulsars(rng: np.random.Generator, count: int, zmax: float = 180.0,
                   wmax: float = 280.0, fmin: float = 5.0, fmax: float = 500.0,
                   snr: tuple = (6.0, 20.0), maxharm: int = 8) -> List[Pulsar]:
    out = []
    for _ in range(count):
        out.append(Pulsar(f=float(rng.uniform(fmin, fmax)),
                          z=float(rng.uniform(-zmax, zmax)),
                          w=float(rng.uniform(-wmax, wmax)),
                          snr=float(rng.uniform(*snr)),
                          nharm=int(rng.integers(1, maxharm + 1)),
                          phase=float(rng.uniform(0, 2 * np.pi))))
    return out


def small_spectrum(seed: int = 20241203):
    """2^20 samples at 64 us (T ~ 67 s) with the single binary pulsar."""
    N, dt = 1 << 20, 64e-6
    ts = timeseries(N, dt, small_pulsar(), seed)
    return presto_fft(ts), N, dt


def red_noise_timeseries(N: int, dt: float, seed: int, pulsars: Sequence[Pulsar] = (),
                         birdies: Sequence[float] = (), birdie_power: float = 400.0,
                         fknee: float = 2.0, slope: float = 1.5, red_level: float = 10.0
                         ) -> np.ndarray:
    """Float32 series for the memory-heavy workload: a white N(0, 1) floor,
    seeded red noise whose power falls as f**-slope below fknee Hz
    (``red_level * ((f / fknee)**-slope - 1)`` times the white level, so it
    meets the floor at the knee), single-bin sinusoids ("birdies") at the
    given frequencies (each rounded to the nearest Fourier bin, normalised
    power ``birdie_power``), and the given pulsars."""
    rng = np.random.default_rng(seed + 1)
    T = N * dt
    nb = N // 2 + 1
    f = np.arange(nb) / T
    shape = np.zeros(nb)
    red = (f > 0) & (f < fknee)
    shape[red] = red_level * ((f[red] / fknee) ** (-slope) - 1.0)
    # E|X_k|^2 = N for unit white noise: the red part has shape * N there
    amp = np.sqrt(shape * N / 2.0)
    X = amp * (rng.standard_normal(nb) + 1j * rng.standard_normal(nb))
    X[0] = 0.0
    X[-1] = 0.0
    # a cosine of amplitude a at integer bin k has X[k] = a N / 2
    a = np.sqrt(4.0 * birdie_power / N)
    for fb in birdies:
        X[int(round(fb * T))] += a * N / 2.0
    x = np.fft.irfft(X, n=N)
    x += timeseries(N, dt, pulsars, seed).astype(np.float64)
    return x.astype(np.float32)


def memory_heavy_birdies() -> List[float]:
    """20 fixed birdie frequencies (Hz): three inside the first rsteps of a
    -flo 1 search at zmax 300 (1.0 - 3.6 Hz), the 50 Hz mains and six of its
    harmonics, and ten scattered ones."""
    return [1.37, 2.11, 3.05, 50.0, 100.0, 150.0, 200.0, 250.0, 300.0, 350.0,
            12.5, 33.3, 61.8, 87.1, 123.0, 177.7, 211.9, 266.6, 404.0, 512.0]


def paper_pulsars(seed: int = 2025) -> List[Pulsar]:
    """Four pulsars: f~U(5,500) Hz, 1-8 harmonics, z~U(-180,180),
    w~U(-280,280), SNR~U(6,20)."""
    return random_pulsars(np.random.default_rng(seed), 4)


# --------------------------------------------------------------------------
# The same construction with torch on any device (the benchmark builds its
# 2^25-sample spectra on the GPU; numpy would take tens of seconds each).

def timeseries_torch(N: int, dt: float, pulsars: Sequence[Pulsar], seed: int, device="cuda"):
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.randn(N, generator=g, device=device, dtype=torch.float64)
    T = N * dt
    u = torch.arange(N, device=device, dtype=torch.float64) / N
    for p in pulsars:
        r = p.f * T
        r0 = r - 0.5 * p.z + p.w / 12.0
        z0 = p.z - 0.5 * p.w
        k = np.arange(1, p.nharm + 1, dtype=np.float64)
        amps = 1.0 / k
        amps = amps * (p.snr / np.sqrt(np.sum(amps ** 2) * N / 4.0))
        phi = u * (r0 + u * (0.5 * z0 + u * (p.w / 6.0)))
        for kk, a in zip(k, amps):
            cyc = kk * phi
            cyc = cyc - torch.floor(cyc)
            x += float(a) * torch.cos(2.0 * np.pi * cyc + p.phase)
    return x.float()


def presto_fft_torch(ts):
    """PRESTO-packed real FFT of a torch series: complex64 tensor of N/2 bins."""
    import torch

    N = ts.shape[0]
    X = torch.fft.rfft(ts.double())
    out = X[: N // 2].to(torch.complex64).clone()
    out[0] = torch.complex(X[0].real, X[N // 2].real).to(torch.complex64)
    return out
