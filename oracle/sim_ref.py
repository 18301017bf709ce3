"""CPU restatement of the signal simulator (numpy).

TEST INFRASTRUCTURE ONLY: the checker of the device simulator
(msosm_gpu_b200/csrc/sim.cu).  Only tests/ import it.

* ``philox4x32_10``: the counter-based generator Philox4x32 with 10 rounds
  (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random
  numbers: as easy as 1, 2, 3", SC11, 2011): per round
  (c0, c1, c2, c3) <- (hi(M1 c2) ^ c1 ^ k0, lo(M1 c2), hi(M0 c0) ^ c3 ^ k1,
  lo(M0 c0)), the key bumped by the Weyl constants between rounds.
* ``normals``: sample i draws one Philox block at counter (i, tag) under the
  key = seed and turns its four words into two complex unit normals by the
  Box-Muller transform in double precision (u1 = (w0 + 1) 2^-32 in (0, 1],
  u2 = w1 2^-32, r = sqrt(-2 ln u1), angle 2 pi u2; likewise w2, w3), each
  component rounded to float32.
* ``emit`` / ``pulsar``: the Gaussian-profile amplitude-modulated pulsar of
  the device simulator, dispersed by the overlap-save filter of the
  reference's design with the +phase chirp (the dispersion filter of
  simulated_pulsar/simulated_complex_signal.cpp:91-120; the filter design
  of dedispersion/overlap_save/osm_prepare.cpp:37-84, oracle
  ``orc_dedisp_params`` with sign +1), in FP64.
* ``quantise_reference``: the reference simulator's uint16 quantisation
  (simulated_complex_signal.cpp:209-228).
"""
from __future__ import annotations

import math

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)
TAG_PULSAR, TAG_AWGN = 0, 1


def philox4x32_10(ctr: np.ndarray, key) -> np.ndarray:
    """ctr: (n, 4) uint32; key: (k0, k1).  Returns (n, 4) uint32."""
    c = [np.asarray(ctr[:, i], np.uint64) for i in range(4)]
    k0, k1 = int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF
    for r in range(10):
        if r:
            k0 = (k0 + W0) & 0xFFFFFFFF
            k1 = (k1 + W1) & 0xFFFFFFFF
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ np.uint64(k0), p1 & MASK,
             (p0 >> np.uint64(32)) ^ c[3] ^ np.uint64(k1), p0 & MASK]
    return np.stack(c, 1).astype(np.uint32)


def blocks(seed: int, start: int, n: int, tag: int) -> np.ndarray:
    i = np.arange(start, start + n, dtype=np.uint64)
    ctr = np.zeros((n, 4), np.uint32)
    ctr[:, 0] = (i & MASK).astype(np.uint32)
    ctr[:, 1] = (i >> np.uint64(32)).astype(np.uint32)
    ctr[:, 2] = tag
    return philox4x32_10(ctr, (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))


def _box_muller(wa: np.ndarray, wb: np.ndarray):
    u1 = (wa.astype(np.float64) + 1.0) * 2.0 ** -32
    u2 = wb.astype(np.float64) * 2.0 ** -32
    r = np.sqrt(-2.0 * np.log(u1))
    a = (2.0 * math.pi) * u2
    return (r * np.cos(a)).astype(np.float32), (r * np.sin(a)).astype(np.float32)


def normals(seed: int, start: int, n: int, tag: int = TAG_PULSAR):
    """Two complex unit normals (unit variance per component) per sample."""
    w = blocks(seed, start, n, tag)
    a0, a1 = _box_muller(w[:, 0], w[:, 1])
    b0, b1 = _box_muller(w[:, 2], w[:, 3])
    z1 = np.empty(n, np.complex64)
    z1.real, z1.imag = a0, a1
    z2 = np.empty(n, np.complex64)
    z2.real, z2.imag = b0, b1
    return z1, z2


def amplitude(t: np.ndarray, bw: float, period: float, fwhm: float, centre: float, snr: float) -> np.ndarray:
    """sqrt(snr g(phase)), g the Gaussian profile of peak 1 and the given FWHM
    (fraction of the period) centred at phase ``centre``; float32."""
    ph = np.mod((t.astype(np.float64) / float(np.float32(bw))) / period, 1.0)
    sig = fwhm / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    d = np.mod(ph - centre + 0.5, 1.0) - 0.5
    g = np.exp(-0.5 * (d / sig) ** 2)
    return np.sqrt(snr * g).astype(np.float32)


def emit(seed, start, n, bw, period, fwhm, centre, snr):
    """The emitted (undispersed) pulsar: amp(t) z1(t) / sqrt(2), and the
    system noise z2(t) / sqrt(2), complex64."""
    z1, z2 = normals(seed, start, n)
    s = np.float32(1.0 / math.sqrt(2.0))
    t = np.arange(start, start + n, dtype=np.int64)
    amp = amplitude(t, bw, period, fwhm, centre, snr)
    e = np.empty(n, np.complex64)
    e.real = (z1.real * s) * amp
    e.imag = (z1.imag * s) * amp
    w = np.empty(n, np.complex64)
    w.real = z2.real * s
    w.imag = z2.imag * s
    return e, w


def osm_filter(x: np.ndarray, H: np.ndarray, M: int) -> np.ndarray:
    """Overlap-save with the reference's H (which carries the factor M):
    y[kM + m] = IFFT_2M(H X_k)[M + m] / (2M)^2, windows x[(k-1)M, (k+1)M),
    zeros before the start (dedispersion/overlap_save/osm_gpu_batch.cpp:94-123)."""
    N = 2 * M
    x = np.asarray(x, np.complex128)
    assert x.size % M == 0
    xp = np.concatenate([np.zeros(M, np.complex128), x])
    out = np.empty(x.size, np.complex128)
    for k in range(x.size // M):
        X = np.fft.fft(xp[k * M:k * M + N])
        y = np.fft.ifft(H * X) * N  # unnormalised inverse
        out[k * M:(k + 1) * M] = y[M:] / (N * N)
    return out


def pulsar(H: np.ndarray, M: int, seed, n, bw, period, fwhm, centre, snr) -> np.ndarray:
    """x = 2 osm(emit) + noise: the dispersed pulsar (the overlap-save output
    is half the normalised convolution) plus the system noise, FP64."""
    e, z2 = emit(seed, 0, n, bw, period, fwhm, centre, snr)
    if H is None:
        return e.astype(np.complex128) + z2
    return 2.0 * osm_filter(e, H, M) + z2


def quantise_reference(v: np.ndarray) -> np.ndarray:
    """(v == 0) ? 0 : uint16(v * 32767 + 32768) per component, float
    arithmetic without contraction, truncation, wrap modulo 2^16
    (simulated_complex_signal.cpp:213-214,225-226)."""
    v = np.asarray(v, np.complex64)
    out = np.empty((v.size, 2), np.uint16)
    for j, comp in enumerate((v.real, v.imag)):
        f = comp.astype(np.float32) * np.float32(32767.0)
        f = (f + np.float32(32768.0)).astype(np.float32)
        q = np.trunc(f).astype(np.int64) & 0xFFFF
        out[:, j] = np.where(comp == 0, 0, q).astype(np.uint16)
    return out
