"""The autotuner on the device: it times every candidate (FFT size x path)
for an observation shape, keeps the fastest, answers a repeated shape from
its cache (also across instances through the cache file), honours the
coherence floor, and its choice dedisperses as the FP64 oracle does within
that path's error budget."""
import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import Dedisperser
from msosm_gpu_b200 import autotune as A

pytestmark = pytest.mark.gpu

BW, F0 = 16e6, 1242e6


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def test_tuner_keeps_the_fastest_candidate_and_caches_it(tmp_path):
    dms = np.linspace(0.0, 60.0, 16)
    path = str(tmp_path / "tune.json")
    t = A.Autotuner(cache_path=path, sample=1 << 20, calls=1)
    ch = t.tune(BW, dms, F0, period=0.0031, time_bin=256)
    cands = A.candidates(BW, dms, F0)
    assert (ch.fftpoint, ch.precision) in cands
    timed = {(r["fftpoint"], r["precision"]): r["ms_per_msample"] for r in t.log}
    assert set(timed) == set(cands)
    assert all(v > 0 for v in timed.values())
    assert ch.ms_per_msample == min(timed.values())
    # a repeated shape is answered from the cache, without timing
    n_log = len(t.log)
    assert t.tune(BW, dms, F0, period=0.0031, time_bin=256) == ch
    assert len(t.log) == n_log
    # and so is a new tuner reading the same cache file
    t2 = A.Autotuner(cache_path=path, sample=1 << 20, calls=1)
    assert t2.tune(BW, dms, F0, period=0.0031, time_bin=256) == ch
    assert not t2.log


def test_tuner_honours_the_coherence_floor():
    dms = np.linspace(0.0, 100.0, 8)
    t = A.Autotuner(sample=1 << 20, calls=1)
    ch = t.tune(BW, dms, F0, period=0.0031, time_bin=256, min_coherence=0.97)
    assert A.coherence(BW, 100.0, F0, ch.fftpoint) >= 0.97
    assert all(A.coherence(BW, 100.0, F0, r["fftpoint"]) >= 0.97 for r in t.log)


def test_tuned_configuration_matches_oracle():
    dms = [0.0, 20.0, 45.0]
    t = A.Autotuner(sample=1 << 20, calls=1)
    ch = t.tune(BW, dms, F0, period=0.0031, time_bin=256)
    count, calls = max(1, 16384 // ch.fftpoint), 3
    d = Dedisperser(BW, dms, F0, ch.fftpoint, count, precision=ch.precision)
    o = O.Dedisp(BW, dms, F0, ch.fftpoint, count)
    rng = np.random.default_rng(3)
    tol = 1.5e-3 if ch.precision == "fp16" else (1e-2 if ch.precision == "bf16" else 2e-5)
    for _ in range(calls):
        x = ((rng.standard_normal(d.block_samples) + 1j * rng.standard_normal(d.block_samples)) * 300).astype(
            np.complex64)
        d.filter_block(x)
        y = d.get_output()
        ref = o.filter(x.astype(np.complex128))
        for i in range(len(dms)):
            assert rel_rms(y[i], ref[i]) < tol, (ch, dms[i], rel_rms(y[i], ref[i]))
