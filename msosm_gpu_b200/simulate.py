"""Seeded synthetic pulsar baseband (host, numpy/scipy).

The reference's SimulatedComplexSignal (simulated_pulsar/
simulated_complex_signal.cpp:40-236) makes two delta spikes per period; the
workloads measured here need a noisy pulsar instead:

  x[t] = disperse( sqrt(snr * g(phase(t))) * n1[t] ) + n2[t]

n1, n2 independent unit-variance complex Gaussian noise (variance 1/2 per
component), g a Gaussian pulse profile of peak 1 and the given FWHM (as a
fraction of the period), so the per-sample pulsar/noise power ratio peaks at
``snr``.  Dispersion applies exp(+i phi(f)) with the same chirp phase as the
dedispersion filter, phi = 2 pi kdm DM f^2 / (f0^2 (f0 + f)), f the offset
from the lower band edge f0 (the sign convention of the reference's
simulator, simulated_complex_signal.cpp:243-251), by overlap-save with
FFTs much longer than the dispersion smear.
"""
from __future__ import annotations

import math

import numpy as np

try:
    import scipy.fft as _fft

    def _fwd(x):
        return _fft.fft(x, workers=-1)

    def _inv(x):
        return _fft.ifft(x, workers=-1)
except ImportError:  # pragma: no cover
    _fwd, _inv = np.fft.fft, np.fft.ifft

KDM = 4.15e15


def smear_samples(bw: float, dm: float, f0: float) -> int:
    return int(math.floor(KDM * dm * (1.0 / f0 ** 2 - 1.0 / (f0 + bw) ** 2) * bw))


def dispersion_phase(nfft: int, bw: float, dm: float, f0: float) -> np.ndarray:
    """phi at the FFT bins of an nfft-point transform of baseband sampled at
    bw: bin k is the offset (k mod nfft)*bw/nfft from the band centre."""
    k = np.arange(nfft, dtype=np.float64)
    off_c = np.where(k < nfft // 2, k, k - nfft) * (bw / nfft)
    f = off_c + bw / 2.0  # offset from the lower edge, in [0, bw)
    return 2.0 * np.pi * KDM * dm * f * f / (f0 * f0 * (f0 + f))


def profile_gaussian(phase: np.ndarray, fwhm: float, centre: float = 0.5) -> np.ndarray:
    sig = fwhm / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    d = (phase - centre + 0.5) % 1.0 - 0.5
    return np.exp(-0.5 * (d / sig) ** 2)


def disperse(x: np.ndarray, bw: float, dm: float, f0: float, nfft: int = 0) -> np.ndarray:
    """Linear (not circular) convolution with the dispersion chirp."""
    nd = smear_samples(bw, dm, f0)
    if nd == 0:
        return x.copy()
    guard = nd + 64
    if nfft == 0:
        nfft = 1 << max(16, int(math.ceil(math.log2(8 * guard))))
    step = nfft - 2 * guard
    Hd = np.exp(1j * dispersion_phase(nfft, bw, dm, f0)).astype(np.complex64)
    n = x.size
    xp = np.concatenate([np.zeros(guard, np.complex64), x.astype(np.complex64),
                         np.zeros(guard + step, np.complex64)])
    out = np.empty(n, np.complex64)
    for s in range(0, n, step):
        seg = xp[s:s + nfft]
        if seg.size < nfft:
            seg = np.concatenate([seg, np.zeros(nfft - seg.size, np.complex64)])
        y = _inv(_fwd(seg) * Hd)
        m = min(step, n - s)
        out[s:s + m] = y[guard:guard + m]
    return out


def pulsar_baseband(n: int, bw: float, f0: float, dm: float, period: float, fwhm: float, snr: float,
                    seed: int = 0, dtype=np.complex64) -> np.ndarray:
    """n samples of amplitude-modulated noise at DM ``dm`` plus system noise
    (see the module docstring).  f0 = lower band edge in Hz."""
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64) / bw
    g = profile_gaussian((t / period) % 1.0, fwhm)
    amp = np.sqrt(snr * g).astype(np.float32)
    s = 1.0 / math.sqrt(2.0)
    n1 = (rng.standard_normal(n, np.float32) + 1j * rng.standard_normal(n, np.float32)) * np.float32(s)
    n2 = (rng.standard_normal(n, np.float32) + 1j * rng.standard_normal(n, np.float32)) * np.float32(s)
    x = disperse((amp * n1).astype(np.complex64), bw, dm, f0) + n2.astype(np.complex64)
    return x.astype(dtype)


def quantise_uint16(x: np.ndarray, scale: float = 1000.0) -> np.ndarray:
    """Offset-binary uint16 pairs (0 reserved for blank), clipped to 1..65535."""
    v = np.empty((x.size, 2), np.float64)
    v[:, 0] = np.rint(x.real * scale) + 32768
    v[:, 1] = np.rint(x.imag * scale) + 32768
    return np.clip(v, 1, 65535).astype(np.uint16)


def dm_grid(n: int, lo: float, hi: float) -> np.ndarray:
    return np.linspace(lo, hi, n).astype(np.float32)
