"""GPU parity against the reference's OWN GPU path: its MSOSM_GPU_DM_concurrent,
MSOSM_GPU_BATCH and OSM_GPU_BATCH classes (cuFFT + its SIMT kernels),
compiled from the reference sources for sm_100a into oracle/_ref/ref_gpu_runner
and run as a separate process on the same seeded uint16 input.

Bar (the plain FP32 path against the reference's cuFFT path): dedispersed
series within 1e-4 relative RMS per trial.  Skipped when the runner was not
built (it needs the reference checkout at build time).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import Dedisperser

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(O.REF_GPU_RUNNER), reason="reference runner not built")]

BW, F0 = 16e6, 1242e6
RTOL = 1e-4


def u16_noise(n, seed, sigma=1000.0):
    rng = np.random.default_rng(seed)
    v = np.clip(np.rint(rng.standard_normal((n, 2)) * sigma) + 32768, 1, 65535)
    return v.astype(np.uint16)


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def run_ref(args, inp):
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.u16"), os.path.join(td, "out.bin")
        inp.tofile(fin)
        a = [str(v) for v in args]
        a = [fin if v == "IN" else fout if v == "OUT" else v for v in a]
        r = subprocess.run([O.REF_GPU_RUNNER] + a, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        return O.read_records(fout)


def ours(dms, fftpoint, count, x_u16, calls, osm=False, precision="fp32"):
    d = Dedisperser(BW, dms, F0, fftpoint, count, osm=osm, precision=precision)
    blk = d.block_samples
    out = []
    for c in range(calls):
        d.filter_block(x_u16[c * blk:(c + 1) * blk])
        out.append(d.get_output())
    return np.concatenate(out, axis=1), d


@pytest.mark.parametrize("fftpoint,count,dms", [
    (1024, 4, [1.0, 3.5, 7.0]),
    (4096, 8, [25.0, 50.0, 73.2, 100.0]),
    (8192, 2, [150.0]),
    (16384, 2, [60.0, 300.0]),
])
def test_concurrent_matches_reference_gpu(fftpoint, count, dms):
    calls = 6
    M = fftpoint // 2
    x = u16_noise(count * M * calls, 11)
    r = run_ref(["concurrent", fftpoint, count, calls, BW, F0, "IN", "OUT"] + dms, x)
    assert int(r["M"][0]) == M and int(r["count"][0]) == count
    ref = r["out"].astype(np.float64).view(np.complex128).reshape(calls, len(dms), count * M)
    ref = np.concatenate(list(ref), axis=1)
    y, _ = ours(dms, fftpoint, count, x, calls)
    for i in range(len(dms)):
        assert rel_rms(y[i], ref[i]) < RTOL, (i, rel_rms(y[i], ref[i]))


@pytest.mark.parametrize("fftpoint,count,dms", [(4096, 8, [0.5, 50.0, 73.2, 100.0]), (8192, 4, [150.0, 200.0]),
                                                (16384, 2, [0.5, 90.0, 300.0])])
def test_tensor_core_path_matches_reference_gpu(fftpoint, count, dms):
    # the f16 tensor-core path against the reference's cuFFT path on the
    # same input, within the tensor path's stated series error (1.5e-3)
    calls = 6
    M = fftpoint // 2
    x = u16_noise(count * M * calls, 14)
    r = run_ref(["concurrent", fftpoint, count, calls, BW, F0, "IN", "OUT"] + dms, x)
    ref = r["out"].astype(np.float64).view(np.complex128).reshape(calls, len(dms), count * M)
    ref = np.concatenate(list(ref), axis=1)
    y, d = ours(dms, fftpoint, count, x, calls, precision="fp16")
    assert d.fftpoint == fftpoint
    for i in range(len(dms)):
        assert rel_rms(y[i], ref[i]) < 1.5e-3, (dms[i], rel_rms(y[i], ref[i]))


def test_single_dm_batch_matches_reference_gpu():
    calls, count, fftpoint, dm = 8, 2, 2048, 12.0
    x = u16_noise(count * fftpoint // 2 * calls, 12)
    r = run_ref(["batch", fftpoint, count, calls, BW, dm, F0, "IN", "OUT"], x)
    ref = r["out"].astype(np.float64).view(np.complex128)
    y, _ = ours([dm], fftpoint, count, x, calls)
    assert rel_rms(y[0], ref) < RTOL


def test_osm_batch_matches_reference_gpu():
    calls, count, dm = 5, 3, 0.5
    d = Dedisperser(BW, [dm], F0, 0, count, osm=True)
    x = u16_noise(d.block_samples * calls, 13)
    r = run_ref(["osm", 0, count, calls, BW, dm, F0, "IN", "OUT"], x)
    assert int(r["M"][0]) == d.M
    ref = r["out"].astype(np.float64).view(np.complex128)
    y, _ = ours([dm], 0, count, x, calls, osm=True)
    assert rel_rms(y[0], ref) < RTOL


@pytest.mark.parametrize("precision,tol", [("fp32", RTOL), ("fp16", 1.5e-3)])
def test_bench_scale_256_trials_match_reference_gpu(precision, tol):
    # the bench's trial grid (256 trials over DM 0-100; the reference cannot
    # run DM 0, so (0, 100]) at FFT 4096 in calls of 32 blocks, as its
    # batch-32 speed test runs them (test_processing_speed_msosm_batch32_dm0to100.cpp)
    calls, count, fftpoint, n = 3, 32, 4096, 256
    M = fftpoint // 2
    dms = [float(v) for v in ((np.arange(n) + 1) * 100.0 / n).astype(np.float32)]
    x = u16_noise(count * M * calls, 21)
    r = run_ref(["concurrent", fftpoint, count, calls, BW, F0, "IN", "OUT"] + [repr(v) for v in dms], x)
    ref = r["out"].view(np.complex64).reshape(calls, n, count * M)
    d = Dedisperser(BW, dms, F0, fftpoint, count, precision=precision)
    worst = 0.0
    for c in range(calls):
        d.filter_block(x[c * count * M:(c + 1) * count * M])
        y = d.get_output()
        for i in range(n):
            worst = max(worst, rel_rms(y[i].astype(np.complex128), ref[c, i].astype(np.complex128)))
    d.close()
    assert worst < tol, worst
