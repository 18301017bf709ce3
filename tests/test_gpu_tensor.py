"""Tensor-core (tcgen05) inverse transforms, MSOSM_FLAG_TENSOR_F16: each GEMM
of the kernel on known data, then the dedispersed series and folded profiles
against the FP64 oracle and against the FP32 CUDA-core path.

Error budget (stated, not tuned): f16 operands carry a relative rounding of
2^-11 at four places (gathered products, DFT constants, twiddled
intermediates, second DFT constants), which gives a series error near 5e-4
relative RMS; the tests bound it at 1.5e-3.  bf16 (2^-8 rounding) gives about
eight times that; bound 1e-2.  Folded profiles average many samples per bin
and are bound at 1e-4 (f16); with bf16 the rounded DFT constants leave a
systematic gain error that averaging does not remove (measured 1.5e-3 here),
bound 5e-3."""
import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import Dedisperser
from msosm_gpu_b200.dedisp import tc_gemm_check

pytestmark = pytest.mark.gpu

BW, F0 = 16e6, 1242e6
SERIES_TOL = 1.5e-3
FOLD_TOL = 1e-4
TOL = {"fp16": (SERIES_TOL, FOLD_TOL), "bf16": (1e-2, 5e-3)}


def rel_rms(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def dft_operand(step):
    """The real form of the inverse DFT the kernel multiplies by, K x N with
    K = [Re | Im] of the input index, rounded to float16: step 1 the 64-point
    DFT, step 2 its frequencies 32..63, step 3 the 128-point DFT, step 4 its
    frequencies 64..127 (FFT 16384's second GEMM)."""
    p = 128 if step >= 3 else 64
    k = np.arange(p)[:, None]
    m = {2: np.arange(32, 64), 4: np.arange(64, 128)}.get(step, np.arange(p))[None, :]
    ang = 2 * np.pi * ((k * m) % p) / p
    c, s = np.cos(ang), np.sin(ang)
    B = np.block([[c, s], [-s, c]])
    return B.astype(np.float16).astype(np.float64)


@pytest.mark.parametrize("step", [1, 2, 3, 4])
def test_gemm_layout_and_readback(step):
    rng = np.random.default_rng(step)
    a = rng.standard_normal((128, 256 if step >= 3 else 128)).astype(np.float16)
    d = tc_gemm_check(step, a)
    ref = a.astype(np.float64) @ dft_operand(step)
    err = np.max(np.abs(d - ref)) / np.max(np.abs(ref))
    assert err < 1e-3, err


def u16(n, seed, scale=1000.0):
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.standard_normal((n, 2)) * scale) + 32768, 1, 65535).astype(np.uint16)


def run_pair(dms, count, calls, seed=0, series=True, x=None, precision="fp16", fft=4096):
    d = Dedisperser(BW, dms, F0, fft, count, precision=precision, series=series)
    o = O.Dedisp(BW, dms, F0, fft, count)
    if x is None:
        x = u16(d.block_samples * calls, seed)
    ours, ref = [], []
    for c in range(calls):
        blk = x[c * d.block_samples:(c + 1) * d.block_samples]
        d.filter_block(blk)
        ours.append(d.get_output())
        ref.append(o.filter(O.decode_uint16(blk)))
    return np.concatenate(ours, 1), np.concatenate(ref, 1), d, x


@pytest.mark.parametrize("precision", ["fp16", "bf16"])
@pytest.mark.parametrize("count,calls", [(6, 3), (5, 4), (1, 5)])
def test_series_matches_oracle(count, calls, precision):
    # DM 0 (no delay), short delays (warm ring after a few blocks) and long
    # ones (blocks before the stream start read as zero); odd counts leave
    # the last block of a call unpaired
    dms = [0.0, 2.0, 5.0, 40.0, 100.0]
    ours, ref, _, _ = run_pair(dms, count, calls, seed=count, precision=precision)
    for i in range(len(dms)):
        e = rel_rms(ours[i], ref[i])
        assert e < TOL[precision][0], (dms[i], e)


@pytest.mark.parametrize("precision", ["fp16", "bf16"])
@pytest.mark.parametrize("count,calls", [(4, 3), (3, 4)])
def test_series_8192_matches_oracle(count, calls, precision):
    # the 8192-point shape: 128-point GEMM 1, one GEMM 2 per block, 16 warps
    dms = [0.0, 5.0, 60.0, 200.0]
    ours, ref, d, _ = run_pair(dms, count, calls, seed=30 + count, precision=precision, fft=8192)
    assert d.fftpoint == 8192
    for i in range(len(dms)):
        e = rel_rms(ours[i], ref[i])
        assert e < TOL[precision][0], (dms[i], e)


@pytest.mark.parametrize("precision", ["fp16", "bf16"])
@pytest.mark.parametrize("count,calls", [(3, 3), (2, 4), (1, 4)])
def test_series_16384_matches_oracle(count, calls, precision):
    # the 16384-point shape: 128 x 128 factorisation, one block per step
    # (both halves of its row), GEMM 2's constant from GEMM 1's columns
    dms = [0.0, 5.0, 60.0, 200.0]
    ours, ref, d, _ = run_pair(dms, count, calls, seed=50 + count, precision=precision, fft=16384)
    assert d.fftpoint == 16384
    for i in range(len(dms)):
        e = rel_rms(ours[i], ref[i])
        assert e < TOL[precision][0], (dms[i], e)


@pytest.mark.parametrize("fft", [8192, 16384])
def test_series_matches_fp32_path_large(fft):
    dms = list(np.linspace(0, 150, 12))
    count, calls = 65536 // fft, 3
    t = Dedisperser(BW, dms, F0, fft, count, precision="fp16")
    f = Dedisperser(BW, dms, F0, fft, count)
    x = u16(t.block_samples * calls, 12)
    for c in range(calls):
        blk = x[c * t.block_samples:(c + 1) * t.block_samples]
        t.filter_block(blk)
        f.filter_block(blk)
        a, b = t.get_output(), f.get_output()
        for i in range(len(dms)):
            assert rel_rms(a[i], b[i]) < SERIES_TOL


def test_series_matches_fp32_path():
    dms = list(np.linspace(0, 100, 16))
    count, calls = 8, 3
    t = Dedisperser(BW, dms, F0, 4096, count, precision="fp16")
    f = Dedisperser(BW, dms, F0, 4096, count)
    x = u16(t.block_samples * calls, 11)
    for c in range(calls):
        blk = x[c * t.block_samples:(c + 1) * t.block_samples]
        t.filter_block(blk)
        f.filter_block(blk)
        a, b = t.get_output(), f.get_output()
        for i in range(len(dms)):
            assert rel_rms(a[i], b[i]) < SERIES_TOL


def test_zero_input_gives_zero():
    d = Dedisperser(BW, [0.0, 50.0], F0, 4096, 4, precision="fp16")
    x = np.full((d.block_samples, 2), 32768, np.uint16)
    for _ in range(2):
        d.filter_block(x)
        assert not np.any(d.get_output())


def test_full_scale_tone_stays_finite_and_accurate():
    # a full-scale tone concentrates the spectrum in one bin: the per-block
    # power-of-two scale must keep every f16 operand in range
    d = Dedisperser(BW, [0.0, 30.0], F0, 4096, 4, precision="fp16")
    o = O.Dedisp(BW, [0.0, 30.0], F0, 4096, 4)
    n = d.block_samples * 3
    t = np.arange(n)
    z = 32000 * np.exp(2j * np.pi * 0.1234 * t)
    x = np.stack([np.rint(z.real) + 32768, np.rint(z.imag) + 32768], 1).astype(np.uint16)
    ours, ref = [], []
    for c in range(3):
        blk = x[c * d.block_samples:(c + 1) * d.block_samples]
        d.filter_block(blk)
        ours.append(d.get_output())
        ref.append(o.filter(O.decode_uint16(blk)))
    ours, ref = np.concatenate(ours, 1), np.concatenate(ref, 1)
    assert np.all(np.isfinite(ours))
    for i in range(2):
        assert rel_rms(ours[i], ref[i]) < SERIES_TOL


@pytest.mark.parametrize("precision,fft", [("fp16", 4096), ("bf16", 4096), ("fp16", 8192), ("fp16", 16384)])
def test_fold_matches_oracle(precision, fft):
    dms, count, calls, period, tb = [0.0, 20.0, 73.2], 8 * 4096 // fft, 6, 0.0011, 256
    d = Dedisperser(BW, dms, F0, fft, count, series=False, precision=precision)
    nd = 4096
    d.fold_init(period, BW, time_bin=tb, discard_Nd=nd)
    o = O.Dedisp(BW, dms, F0, fft, count)
    x = u16(d.block_samples * calls, 21)
    ser = []
    for c in range(calls):
        blk = x[c * d.block_samples:(c + 1) * d.block_samples]
        d.filter_block(blk)
        ser.append(o.filter(O.decode_uint16(blk)))
    ser = np.concatenate(ser, 1)
    prof = d.get_profiles()
    assert d.folded_periods() > 0
    for i in range(len(dms)):
        f = O.Fold(period, BW, d.block_samples, tb)
        f.discard_samples(nd)
        for c in range(calls):
            f.fold_data(np.abs(ser[i, c * d.block_samples:(c + 1) * d.block_samples]) ** 2)
        e = rel_rms(prof[i], f.fold_data_bins())
        assert e < TOL[precision][1], (dms[i], e)


@pytest.mark.parametrize("fft,period,tb", [(8192, 0.0011, 4096), (16384, 0.0011, 4096), (4096, 0.0008, 1024),
                                           (16384, 0.0008, 1024)])
def test_fold_short_bins(fft, period, tb):
    # 4096 bins of 4 samples: above the 2048 bins the 8192 and 16384 kernels
    # keep in shared memory (the work items' partial rows live in global
    # memory) and below 8 samples per bin (each block goes span piece by span
    # piece); 1024 bins of 12 samples: the 8-samples-per-thread fast path of
    # a block instead of the one-pass fold of a step (>= 16 samples per bin)
    dms, count, calls = [0.0, 30.0], 65536 // fft, 4
    d = Dedisperser(BW, dms, F0, fft, count, series=False, precision="fp16")
    nd = 4096
    d.fold_init(period, BW, time_bin=tb, discard_Nd=nd)
    o = O.Dedisp(BW, dms, F0, fft, count)
    x = u16(d.block_samples * calls, 27)
    ser = []
    for c in range(calls):
        blk = x[c * d.block_samples:(c + 1) * d.block_samples]
        d.filter_block(blk)
        ser.append(o.filter(O.decode_uint16(blk)))
    ser = np.concatenate(ser, 1)
    prof = d.get_profiles()
    assert prof.shape == (len(dms), tb) and d.folded_periods() > 0
    for i in range(len(dms)):
        f = O.Fold(period, BW, d.block_samples, tb)
        f.discard_samples(nd)
        for c in range(calls):
            f.fold_data(np.abs(ser[i, c * d.block_samples:(c + 1) * d.block_samples]) ** 2)
        # 4 or 12 samples per bin average little: the bound is the series one
        assert rel_rms(prof[i], f.fold_data_bins()) < SERIES_TOL, dms[i]


@pytest.mark.parametrize("precision,fft,detect", [("fp16", 4096, "power"), ("fp16", 8192, "power"),
                                                  ("fp16", 4096, "amplitude"), ("bf16", 8192, "power"),
                                                  ("fp16", 16384, "power"), ("fp16", 16384, "amplitude")])
def test_series_and_fold_in_one_pass(precision, fft, detect):
    # the kernel that writes the series and folds in the same pass: both
    # outputs against the oracle, |y| as well as |y|^2 detection
    dms, count, calls, period, tb = [0.0, 20.0, 73.2], 8 * 4096 // fft, 6, 0.0011, 256
    d = Dedisperser(BW, dms, F0, fft, count, series=True, precision=precision)
    nd = 4096
    d.fold_init(period, BW, time_bin=tb, discard_Nd=nd, detect=detect)
    o = O.Dedisp(BW, dms, F0, fft, count)
    x = u16(d.block_samples * calls, 23)
    ours, ser = [], []
    for c in range(calls):
        blk = x[c * d.block_samples:(c + 1) * d.block_samples]
        d.filter_block(blk)
        ours.append(d.get_output())
        ser.append(o.filter(O.decode_uint16(blk)))
    ours, ser = np.concatenate(ours, 1), np.concatenate(ser, 1)
    prof = d.get_profiles()
    assert d.folded_periods() > 0
    for i in range(len(dms)):
        assert rel_rms(ours[i], ser[i]) < TOL[precision][0], dms[i]
        f = O.Fold(period, BW, d.block_samples, tb)
        f.discard_samples(nd)
        for c in range(calls):
            y = ser[i, c * d.block_samples:(c + 1) * d.block_samples]
            f.fold_data(np.abs(y) if detect == "amplitude" else np.abs(y) ** 2)
        assert rel_rms(prof[i], f.fold_data_bins()) < TOL[precision][1], dms[i]


def test_complex64_device_input_matches_uint16_host_input():
    # the bench feeds complex64 already on the device; the same values as
    # offset-binary host pairs give bit-identical series
    import torch
    dms, count, calls = [0.0, 30.0, 90.0], 4, 3
    a = Dedisperser(BW, dms, F0, 4096, count, precision="fp16")
    b = Dedisperser(BW, dms, F0, 4096, count, precision="fp16")
    bs = a.block_samples
    x = u16(bs * calls, 31)
    xd = torch.from_numpy(O.decode_uint16(x).astype(np.complex64)).cuda()
    for c in range(calls):
        a.filter_block(x[c * bs:(c + 1) * bs])
        b.filter_block(xd[c * bs:(c + 1) * bs])
        assert np.array_equal(a.get_output(), b.get_output())


@pytest.mark.parametrize("fftpoint", [4096, 8192, 16384])
def test_wait_timeout_reports_and_handle_recovers(fftpoint):
    # a wait limit of 0 makes the kernel's first wait on a GEMM give up: it
    # takes its timeout exit (status word, drain of its own GEMMs, tensor
    # memory freed) without hanging, the next synchronising call reports
    # MSOSM_ERR_TIMEOUT, and after the default limit is restored the handle
    # dedisperses its later calls exactly as the oracle does
    from msosm_gpu_b200 import _abi
    dms, count, calls = [10.0, 60.0], 6, 5
    d = Dedisperser(BW, dms, F0, fftpoint, count, precision="fp16")
    o = O.Dedisp(BW, dms, F0, fftpoint, count)
    xs = [O.decode_uint16(u16(d.block_samples, 40 + c)).astype(np.complex64) for c in range(calls)]
    d.filter_block(xs[0])
    o.filter(xs[0].astype(np.complex128))
    d.get_output()
    d.set_tc_wait_limit(0)
    d.filter_block(xs[1])
    o.filter(xs[1].astype(np.complex128))
    with pytest.raises(_abi.MsosmError) as ei:
        d.get_output()
    assert ei.value.status == _abi.ERR_TIMEOUT
    d.set_tc_wait_limit(-1)
    for c in range(2, calls):
        d.filter_block(xs[c])
        ref = o.filter(xs[c].astype(np.complex128))
        y = d.get_output()
        for i in range(len(dms)):
            assert rel_rms(y[i], ref[i]) < SERIES_TOL, (c, i)
    with pytest.raises(_abi.MsosmError):
        Dedisperser(BW, dms, F0, fftpoint, count).set_tc_wait_limit(0)
