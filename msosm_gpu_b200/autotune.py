"""Autotuner: the FFT size and inverse-transform path per observation.

For an observation (band, lower edge, DM trials, fold settings) the tuner
times every candidate on the device and keeps the fastest one whose error
against FP64 fits the budget:

* FFT sizes 2^11 .. 2^15 at or above the MS-OSM minimum 2 M_min (smaller
  sizes are raised to it, msosm_gpu_dm_concurrent.cpp:33-35, so they are the
  same candidate);
* the FP32 CUDA-core kernel at every size; the tensor-core kernel at 4096,
  8192 and 16384 with f16 operands (folded-profile error ~2e-5, series ~5e-4) and with
  bf16 operands (profiles ~1.3e-3, series ~4e-3) when the budget admits it.

Each candidate runs `calls` timed filter_block calls (after one warm-up) of
about `sample` samples of device-resident noise, CUDA events on the handle's
stream.  Results are cached per observation shape (and in a JSON file when
``cache_path`` is given).

Every valid size gives the reference's MS-OSM result, but not the same one:
the multi-segment approximation of the dispersion filter tightens as M grows.
Measured against exact coherent dedispersion (classical overlap-save with the
full-length filter) with the FP64 oracle, the coherence of the two outputs is
rho ~ 1 - 0.24 sqrt(Nd) / M: 0.92 at the minimum FFT for 16 MHz at DM 100,
0.875 for 64 MHz at DM 80, the loss halving with each doubling of M.  The
fastest size is the least coherent, so ``min_coherence`` drops the sizes
whose modelled coherence, for the trial of largest Nd, falls below it.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import asdict, dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .dedisp import Dedisperser
from .prepare import msosm_min_order as min_order_msosm, nd

# relative RMS error of the folded profiles against FP64, per path (measured
# on the 64 MHz / FFT 8192 precision sweep and the tensor-core parity tests)
PROFILE_ERROR = {"fp32": 1e-6, "fp16": 3e-5, "bf16": 2e-3}
TENSOR_SIZES = (4096, 8192, 16384)
# 1 - rho = COHERENCE_SLOPE sqrt(Nd) / M, fitted to the FP64 oracle
# (tests/test_msosm_coherence_cpu.py pins it within 25 %)
COHERENCE_SLOPE = 0.24


def coherence(bw: float, dm: float, f0: float, fftpoint: int) -> float:
    """Modelled coherence of MS-OSM at this FFT size with exact coherent
    dedispersion (0 .. 1)."""
    M = int(fftpoint) // 2
    return max(0.0, 1.0 - COHERENCE_SLOPE * math.sqrt(nd(bw, float(dm), f0)) / M)


@dataclass
class Choice:
    fftpoint: int
    precision: str
    ms_per_msample: float  # device ms per million input samples (all trials)


def candidates(bw: float, dms: Sequence[float], f0: float, budget: float = 1e-3,
               sizes: Sequence[int] = tuple(1 << k for k in range(11, 16)),
               min_coherence: Optional[float] = None) -> List[Tuple[int, str]]:
    """(fftpoint, precision) pairs worth timing for these trials; with
    ``min_coherence`` only sizes whose modelled coherence (largest-Nd trial)
    reaches it.  ValueError when no size does."""
    m_min = max(min_order_msosm(nd(bw, float(d), f0)) for d in dms)
    out = []
    ns = sorted(set(max(int(s), 2 * m_min) for s in sizes))
    if min_coherence is not None:
        d_worst = max(float(d) for d in dms)
        ns = [n for n in ns if coherence(bw, d_worst, f0, n) >= min_coherence]
        if not ns:
            raise ValueError(f"no FFT size of {list(sizes)} reaches coherence {min_coherence}")
    for n in ns:
        out.append((n, "fp32"))
        if n in TENSOR_SIZES:
            for p in ("fp16", "bf16"):
                if PROFILE_ERROR[p] <= budget:
                    out.append((n, p))
    return out


def _key(bw, dms, f0, time_bin, budget, sizes, min_coherence=None) -> str:
    d = np.asarray(dms, np.float64)
    return json.dumps([round(float(bw)), round(float(f0)), int(d.size), round(float(d.min()), 4),
                       round(float(d.max()), 4), int(time_bin), budget, list(sizes)]
                      + ([] if min_coherence is None else [min_coherence]))


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, sample: int = 1 << 22, calls: int = 2):
        self.cache_path = cache_path
        self.sample = sample
        self.calls = calls
        self.cache: Dict[str, dict] = {}
        if cache_path and os.path.exists(cache_path):
            self.cache = json.load(open(cache_path))
        self.log: List[dict] = []

    def _time(self, bw, dms, f0, fftpoint, precision, period, time_bin) -> float:
        import torch
        M = fftpoint // 2
        count = max(2, self.sample // M)
        x = torch.randn(count * M, dtype=torch.complex64, device="cuda") * 100
        stream = torch.cuda.Stream()
        d = Dedisperser(bw, dms, f0, fftpoint, count=count, series=False, precision=precision)
        try:
            d.set_stream(stream)
            if period:
                d.fold_init(period, bw, time_bin=time_bin, discard_Nd=int(d.Nd.max()), detect="power")
            d.filter_block(x)
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                s.record(stream)
                for _ in range(self.calls):
                    d.filter_block(x)
                e.record(stream)
            torch.cuda.synchronize()
            return s.elapsed_time(e) / (self.calls * count * M / 1e6)
        finally:
            d.close()

    def tune(self, bw: float, dms: Sequence[float], f0: float, period: float = 0.0, time_bin: int = 1024,
             budget: float = 1e-3, sizes: Sequence[int] = tuple(1 << k for k in range(11, 16)),
             min_coherence: Optional[float] = None) -> Choice:
        key = _key(bw, dms, f0, time_bin, budget, sizes, min_coherence)
        if key in self.cache:
            return Choice(**self.cache[key])
        best = None
        for n, p in candidates(bw, dms, f0, budget, sizes, min_coherence):
            ms = self._time(bw, dms, f0, n, p, period, time_bin)
            self.log.append({"key": key, "fftpoint": n, "precision": p, "ms_per_msample": ms})
            if best is None or ms < best.ms_per_msample:
                best = Choice(n, p, ms)
        self.cache[key] = asdict(best)
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump(self.cache, f)
        return best


def fixed_choice(bw: float, dms: Sequence[float], f0: float, fftpoint: int, precision: str) -> Tuple[int, str]:
    """A fixed configuration applied to one observation: the FFT raised to
    the observation's minimum, the tensor path only where its sizes allow."""
    m_min = max(min_order_msosm(nd(bw, float(d), f0)) for d in dms)
    n = max(int(fftpoint), 2 * m_min)
    if precision != "fp32" and n not in TENSOR_SIZES:
        precision = "fp32"
    return n, precision


def log_uniform(rng, lo: float, hi: float) -> float:
    return float(math.exp(rng.uniform(math.log(lo), math.log(hi))))
