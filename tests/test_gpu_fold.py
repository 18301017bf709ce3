"""Fold_GPU on the device: the standalone fold against the reference's own
Fold_GPU (golden vectors from its host code), and the two-polarisation
pipeline of msosm_psrdada.cpp:105-142 (two MSOSM_GPU_BATCH + Fold_GPU)
against the reference's GPU classes and the oracle."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import Dedisperser, Fold_GPU

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
META = json.load(open(os.path.join(HERE, "golden", "reference_host.json")))
ARR = np.load(os.path.join(HERE, "golden", "reference_host.npz"))
BW, F0 = 16e6, 1242e6


def rel_rms(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, float) - b) ** 2) / np.mean(np.asarray(b, float) ** 2)))


@pytest.mark.parametrize("k", range(len(META["fold"])))
def test_device_fold_matches_reference_fold_gpu(k):
    s = META["fold"][k]
    I = ARR[f"fold{k}_intensity"].astype(np.float32)
    f = Fold_GPU(s["period"], s["fs"], s["size"], time_bin=s["time_bin"])
    assert f.period_samples == s["period_samples"]
    assert f.time_bin == s["time_bin_out"]
    f.discard_samples(s["Nd"])
    for c in range(s["chunks"]):
        f.set_intensity(I[c * s["size"]:(c + 1) * s["size"]])
        f.fold_data()
    np.testing.assert_allclose(f.fold_data_bins(), ARR[f"fold{k}_folded"], rtol=1e-6, atol=1e-6)


def u16(n, seed):
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.standard_normal((n, 2)) * 1000) + 32768, 1, 65535).astype(np.uint16)


def test_two_pol_pipeline_matches_reference_gpu_and_oracle():
    fftpoint, count, dm, period, tb, calls = 2048, 4, 5.0, 0.0011, 32, 24
    a = Dedisperser(BW, [dm], F0, fftpoint, count)
    b = Dedisperser(BW, [dm], F0, fftpoint, count)
    blk = a.block_samples
    xa, xb = u16(blk * calls, 1), u16(blk * calls, 2)
    fold = Fold_GPU(period, BW, blk, time_bin=tb)
    nd = int(a.Nd[0])
    fold.discard_samples(nd)
    for c in range(calls):
        a.filter_block(xa[c * blk:(c + 1) * blk])
        b.filter_block(xb[c * blk:(c + 1) * blk])
        fold.calculate_intensity(a, b)
        fold.fold_data()
    ours = fold.fold_data_bins()
    assert ours.shape == (tb,) and ours.any()
    # oracle: FP64 dedispersion of both pols, sqrt(|a|^2+|b|^2), Fold_GPU state machine
    oa, ob = O.Dedisp(BW, [dm], F0, fftpoint, count), O.Dedisp(BW, [dm], F0, fftpoint, count)
    of = O.Fold(period, BW, blk, tb)
    of.discard_samples(nd)
    for c in range(calls):
        ya = oa.filter(O.decode_uint16(xa[c * blk:(c + 1) * blk]))[0]
        yb = ob.filter(O.decode_uint16(xb[c * blk:(c + 1) * blk]))[0]
        of.fold_data(O.intensity(ya, yb))
    assert rel_rms(ours, of.fold_data_bins()) < 2e-5
    # the reference's own GPU classes
    if not os.path.exists(O.REF_GPU_RUNNER):
        pytest.skip("reference runner not built")
    with tempfile.TemporaryDirectory() as td:
        fa, fb, fo = (os.path.join(td, n) for n in ("a.u16", "b.u16", "o.bin"))
        xa.tofile(fa)
        xb.tofile(fb)
        r = subprocess.run([O.REF_GPU_RUNNER, "fold2", str(fftpoint), str(count), str(calls), str(BW), str(dm),
                            str(F0), str(period), str(tb), fa, fb, fo], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        ref = O.read_records(fo)["folded"]
    assert rel_rms(ours, ref) < 1e-4, rel_rms(ours, ref)


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_fused_fold_with_many_spans_per_call(precision):
    # a 10 us period at 16 MHz (160 samples) over calls of 2^22 samples: about
    # 26k period spans per call, more than the span upload's one pass of
    # 64 x 256 threads, from host inputs over both staging buffers
    dm, fftpoint, count, calls, period, tb = 5.0, 4096, 2048, 2, 1e-5, 16
    d = Dedisperser(BW, [dm], F0, fftpoint, count, series=False, precision=precision)
    blk = d.block_samples
    nd = int(d.Nd[0])
    d.fold_init(period, BW, time_bin=tb, discard_Nd=nd)
    o = O.Dedisp(BW, [dm], F0, fftpoint, count)
    of = O.Fold(period, BW, blk, tb)
    assert blk // of.period_samples > 64 * 256
    of.discard_samples(nd)
    x = u16(blk * calls, 7)
    for c in range(calls):
        part = x[c * blk:(c + 1) * blk]
        d.filter_block(part)
        of.fold_data(np.abs(o.filter(O.decode_uint16(part))[0]) ** 2)
    ours = d.get_profiles()[0]
    assert d.folded_periods() > 2 * 64 * 256
    assert rel_rms(ours, of.fold_data_bins()) < (1e-5 if precision == "fp32" else 1e-4)
