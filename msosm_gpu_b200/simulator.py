"""The signal simulator on the GPU (``msosm_sim_*`` of the C ABI).

* ``normals``: the counter-based complex unit normals every simulator draws
  (Philox4x32-10 + Box-Muller; a sample's numbers depend only on the seed,
  its index and a tag, so chunked and whole-signal generation agree).
* ``AWGN`` and ``SimulatedComplexSignal``: the reference's classes
  (simulated_pulsar/include/AWGN.h:8-31,
  simulated_pulsar/include/simulated_complex_signal.h:9-63) with the same
  constructors, methods and public fields; ``seed`` replaces the reference's
  default-seeded engine.
* ``PulsarSimulator``: a streaming noisy pulsar with a Gaussian profile,
  dispersed through the library's overlap-save path with the dispersion
  filter, for workloads of any length (``pulsar_baseband`` returns a whole
  signal).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _abi
from ._abi import check, lib

TAG_PULSAR = _abi.SIM_TAG_PULSAR
TAG_AWGN = _abi.SIM_TAG_AWGN


def _ptr(a) -> int:
    """Host numpy array or device tensor (anything with data_ptr())."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def normals(seed: int, start: int, n: int, tag: int = TAG_PULSAR):
    """(z1, z2): complex64 unit normals of samples start .. start + n - 1."""
    z1 = np.empty(n, np.complex64)
    z2 = np.empty(n, np.complex64)
    if n:
        check(lib().msosm_sim_normals(seed, start, n, tag, z1.ctypes.data, z2.ctypes.data))
    return z1, z2


class AWGN:
    """AWGN() / AWGN(mean, variance, n) / AWGN(SNR, n) (AWGN.cpp:3-27).
    ``generateNoiseSamples`` returns n complex64 samples: variance used as the
    standard deviation, or sigma / sqrt(2) unit normals, sigma =
    sqrt(10^(-SNR/10)) (AWGN.cpp:29-58)."""

    def __init__(self, *args, seed: int = 0):
        if len(args) == 0:
            self.mean, self.variance, self.numberOfSamples, self.isSNRMode = 0.0, 1.0, 100, False
            self.SNR = 0.0
        elif len(args) == 2:
            self.SNR, self.numberOfSamples = float(args[0]), int(args[1])
            self.mean, self.variance, self.isSNRMode = 0.0, 1.0, True
        elif len(args) == 3:
            self.mean, self.variance, self.numberOfSamples = float(args[0]), float(args[1]), int(args[2])
            self.isSNRMode, self.SNR = False, 0.0
        else:
            raise TypeError("AWGN(), AWGN(mean, variance, n) or AWGN(SNR, n)")
        self.seed = seed
        self.samples = None

    @property
    def sigma(self) -> float:
        return float(np.float32(np.sqrt(10.0 ** float(np.float32(-self.SNR) / np.float32(10)))))

    def generateNoiseSamples(self) -> np.ndarray:
        out = np.empty(self.numberOfSamples, np.complex64)
        if out.size:
            check(lib().msosm_sim_awgn(self.seed, out.size, int(self.isSNRMode), self.mean, self.variance,
                                       self.SNR, out.ctypes.data))
        self.samples = out
        return out

    def deallocate(self) -> None:
        self.samples = None


class SimulatedComplexSignal:
    """SimulatedComplexSignal(bw, dm, f0, period, mode) with
    ``generate_pulsar_signal(repeat, add_noise, SNR)``
    (simulated_complex_signal.cpp:12-236), computed on the GPU.  Public
    fields as the reference: signal (complex64), signal_u16 ((n, 2) uint16
    when mode is "uint16"), data_type, signal_size, Np, Nd, M, M_min, range;
    plus signal_power (dB) and seed."""

    def __init__(self, bw: float, dm: float, f0: float, period: float, mode: str = "complex", seed: int = 0):
        self.bw, self.dm, self.f0, self.period = float(bw), float(dm), float(f0), float(period)
        self.data_type = mode
        self.seed = seed
        info = _abi.SimTwoSpikeInfo()
        check(lib().msosm_sim_two_spike_shape(self.bw, self.dm, self.f0, self.period, ctypes.byref(info)))
        self.Np, self.Nd, self.range, self.order = int(info.Np), int(info.Nd), int(info.range), int(info.order)
        m = ctypes.c_ulong()
        check(lib().msosm_prepare_min_order_msosm(self.Nd, ctypes.byref(m)))
        self.M_min = self.M = int(m.value)
        self.signal = None
        self.signal_u16 = None
        self.signal_size = 0
        self.signal_power = None

    def generate_pulsar_signal(self, repeat: int = 1, add_noise: bool = False, SNR: float = 0.0,
                               pinned: bool = True) -> None:
        self.signal_size = int(repeat) * self.Np
        self.signal = np.empty(self.signal_size, np.complex64)
        self.signal_u16 = np.empty((self.signal_size, 2), np.uint16) if self.data_type == "uint16" else None
        p = ctypes.c_float()
        check(lib().msosm_sim_two_spike(self.bw, self.dm, self.f0, self.period, int(repeat), int(bool(add_noise)),
                                        float(SNR), self.seed, self.signal.ctypes.data,
                                        None if self.signal_u16 is None else self.signal_u16.ctypes.data,
                                        ctypes.byref(p)))
        self.signal_power = float(p.value)


class PulsarSimulator:
    """Streaming noisy pulsar x(t) = D[a z1](t) + z2(t)/sqrt(2) (see
    msosm_sim_pulsar_params in msosm_b200.h): ``next()`` returns the next
    ``chunk`` samples, ``next(u16_scale=s)`` also their offset-binary uint16
    pairs; ``out`` may be a device tensor."""

    def __init__(self, bw: float, f0: float, dm: float, period: float, fwhm: float, snr: float,
                 seed: int = 0, centre: float = 0.5, min_chunk: int = 0):
        p = _abi.SimPulsarParams(bw=bw, f0=f0, dm=dm, period=period, fwhm=fwhm, centre=centre, snr=snr, seed=seed)
        h = ctypes.c_void_p()
        check(lib().msosm_sim_pulsar_create(ctypes.byref(p), int(min_chunk), ctypes.byref(h)))
        self._h = h
        info = _abi.SimPulsarInfo()
        check(lib().msosm_sim_pulsar_get_info(self._h, ctypes.byref(info)))
        self.chunk, self.M, self.Nd = int(info.chunk), int(info.M), int(info.Nd)

    @property
    def next_sample(self) -> int:
        info = _abi.SimPulsarInfo()
        check(lib().msosm_sim_pulsar_get_info(self._h, ctypes.byref(info)))
        return int(info.next_sample)

    def next(self, out=None, u16=None, u16_scale: float = 0.0, want_complex: bool = True):
        """Fills (or allocates on the host) the next chunk; returns (out, u16)."""
        if out is None and want_complex:
            out = np.empty(self.chunk, np.complex64)
        if u16 is None and u16_scale:
            u16 = np.empty((self.chunk, 2), np.uint16)
        check(lib().msosm_sim_pulsar_next(self._h, _ptr(out), _ptr(u16), float(u16_scale)))
        return out, u16

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().msosm_sim_pulsar_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pulsar_baseband(n: int, bw: float, f0: float, dm: float, period: float, fwhm: float, snr: float,
                    seed: int = 0, centre: float = 0.5, device=None, min_chunk: int = 0):
    """The first n samples of a PulsarSimulator stream: a host complex64
    array, or with ``device`` (a torch device) a device tensor."""
    sim = PulsarSimulator(bw, f0, dm, period, fwhm, snr, seed=seed, centre=centre,
                          min_chunk=min_chunk or min(n, 1 << 24))
    try:
        if device is not None:
            import torch
            buf = torch.empty(-(-n // sim.chunk) * sim.chunk, dtype=torch.complex64, device=device)
            for c in range(0, buf.numel(), sim.chunk):
                sim.next(out=buf[c:c + sim.chunk])
            return buf[:n]
        out = np.empty(-(-n // sim.chunk) * sim.chunk, np.complex64)
        for c in range(0, out.size, sim.chunk):
            sim.next(out=out[c:c + sim.chunk])
        return out[:n]
    finally:
        sim.close()
