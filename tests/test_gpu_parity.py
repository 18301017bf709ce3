"""GPU parity: the sm_100a path through the C ABI against the FP64 oracle
(oracle/orc.c) on the same seeded inputs.

Tolerances: the FP32 path must stay within 2e-5 relative RMS of the FP64
restatement per DM trial (the bar for the reference's own cuFFT path is
1e-4); folded profiles within 2e-5 relative RMS.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import Dedisperser, MsosmError, prepare

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
RTOL_SERIES = 2e-5
RTOL_FOLD = 2e-5
BW, F0 = 16e6, 1242e6


def noise(n, seed, scale=100.0):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64) * np.float32(scale)


def u16_noise(n, seed, sigma=1000.0):
    rng = np.random.default_rng(seed)
    v = np.clip(np.rint(rng.standard_normal((n, 2)) * sigma) + 32768, 1, 65535)
    return v.astype(np.uint16)


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / max(np.mean(np.abs(b) ** 2), 1e-300)))


def run_pair(dms, fftpoint, count, calls, seed=0, osm=False, kind="c64", bw=BW, f0=F0):
    d = Dedisperser(bw, dms, f0, fftpoint, count, osm=osm)
    o = O.Dedisp(bw, dms, f0, fftpoint, count, osm=osm)
    assert (d.M, d.count) == (o.M, o.count)
    assert list(d.delaycount) == o.delaycount
    ours, ref = [], []
    for c in range(calls):
        if kind == "c64":
            x = noise(d.block_samples, seed + c)
            xo = x.astype(np.complex128)
        else:
            x = u16_noise(d.block_samples, seed + c)
            xo = O.decode_uint16(x)
        d.filter_block(x)
        ours.append(d.get_output())
        ref.append(o.filter(xo))
    return np.concatenate(ours, axis=1), np.concatenate(ref, axis=1), d


@pytest.mark.parametrize("fftpoint,dms", [
    (1024, [0.5, 3.0, 5.0, 7.5]),
    (4096, [10.0, 50.0, 73.2]),
    (512, [0.25, 1.0, 1.9]),
    (2048, [20.0, 25.0]),
    (8192, [100.0, 150.0]),
    (16384, [300.0]),
    (256, [0.1, 0.3]),
])
def test_msosm_series_matches_oracle(fftpoint, dms):
    ours, ref, _ = run_pair(dms, fftpoint, count=4, calls=5)
    for i in range(len(dms)):
        assert rel_rms(ours[i], ref[i]) < RTOL_SERIES, (i, rel_rms(ours[i], ref[i]))


def test_msosm_count1_many_calls_ring_wraps():
    ours, ref, d = run_pair([2.0, 6.0], 1024, count=1, calls=40)
    assert d.ring_slots < 40
    for i in range(2):
        assert rel_rms(ours[i], ref[i]) < RTOL_SERIES


def test_msosm_uint16_input():
    ours, ref, _ = run_pair([1.0, 4.0, 8.0], 1024, count=8, calls=4, kind="u16")
    for i in range(3):
        assert rel_rms(ours[i], ref[i]) < RTOL_SERIES


def test_dm_zero_trial_is_a_pure_overlap_save():
    ours, ref, d = run_pair([0.0, 3.0], 1024, count=4, calls=4)
    assert d.delaycount[0] == 0
    for i in range(2):
        assert rel_rms(ours[i], ref[i]) < RTOL_SERIES


def test_osm_matches_oracle():
    ours, ref, d = run_pair([0.5, 0.25], 0, count=3, calls=4, osm=True)
    assert d.fftpoint == 4096
    for i in range(2):
        assert rel_rms(ours[i], ref[i]) < RTOL_SERIES


def test_count_invariance_of_the_stream():
    # the output stream must not depend on how the input is cut into calls
    x = noise(1024 * 16, 99)
    outs = []
    for count in (1, 4, 16):
        d = Dedisperser(BW, [3.0, 7.0], F0, 2048, count)
        blk = d.block_samples
        res = []
        for c in range(x.size // blk):
            d.filter_block(x[c * blk:(c + 1) * blk])
            res.append(d.get_output())
        outs.append(np.concatenate(res, axis=1))
    for o in outs[1:]:
        assert rel_rms(o, outs[0]) < 1e-6


def test_uint16_output_codec_matches_oracle_encoding():
    d = Dedisperser(BW, [2.0, 5.0], F0, 1024, 4)
    x = u16_noise(d.block_samples, 5, sigma=3000)
    d.filter_block(x)
    y = d.get_output()
    u = d.get_output(dtype=np.uint16)
    # encoding rule of complexToUint16: uint16(v + 32768*(v != 0)), truncating
    re, im = y.real.astype(np.float32), y.imag.astype(np.float32)
    er = np.clip(re + np.where(re != 0, 32768.0, 0.0).astype(np.float32), 0, 65535).astype(np.uint16)
    ei = np.clip(im + np.where(im != 0, 32768.0, 0.0).astype(np.float32), 0, 65535).astype(np.uint16)
    np.testing.assert_array_equal(u[..., 0], er)
    np.testing.assert_array_equal(u[..., 1], ei)


def test_reference_layout_with_trailing_element():
    d = Dedisperser(BW, [2.0, 5.0], F0, 1024, 2)
    d.filter_block(noise(d.block_samples, 1))
    out = np.full(2 * d.block_samples + 1, 7 + 7j, np.complex64)
    d.get_output(out=out)
    assert out[-1] == 0
    np.testing.assert_array_equal(out[:-1].reshape(2, -1), d.get_output())


def test_filter_design_on_device_matches_reference_golden():
    meta = json.load(open(os.path.join(HERE, "golden", "reference_host.json")))
    arr = np.load(os.path.join(HERE, "golden", "reference_host.npz"))
    for k, s in enumerate(meta["msosm"]):
        if 2 * s["M"] < 64 or 2 * s["M"] > 16384:
            continue
        H = prepare.dedisp_params(s["bw"], s["dm"], s["f0"], s["M"])
        Hr = arr[f"msosm{k}_H"].astype(np.float64).view(np.complex128)
        assert rel_rms(H, Hr) < 2e-5, (k, rel_rms(H, Hr))
        Ho = O.dedisp_params(s["bw"], s["dm"], s["f0"], s["M"])
        assert rel_rms(H, Ho) < 2e-5


def test_handle_parameters_match_reference_prepare():
    d = Dedisperser(BW, [50.0, 73.2], F0, 4096, 2)
    for i, dm in enumerate([50.0, 73.2]):
        dc, dp = O.segmentation(BW, dm, F0, d.M)
        np.testing.assert_array_equal(d.delay_points(i), dp)
        assert rel_rms(d.dedisp_params(i), O.dedisp_params(BW, dm, F0, d.M)) < 2e-5


def _fold_oracle(series, period, fs, time_bin, Nd, detect):
    out = []
    for row in series:
        f = O.Fold(period, fs, row.size // NCALLS_FOLD, time_bin, accumulate_float=False)
        f.discard_samples(Nd)
        inten = np.abs(row) if detect == "amplitude" else np.abs(row) ** 2
        for c in range(NCALLS_FOLD):
            n = row.size // NCALLS_FOLD
            f.fold_data(inten[c * n:(c + 1) * n])
        out.append(f.fold_data_bins())
    return np.array(out)


NCALLS_FOLD = 24


@pytest.mark.parametrize("detect,time_bin,period", [
    ("amplitude", 32, 0.00123),
    ("power", 0, 0.000317),
    ("power", 64, 0.00031),
])
def test_fused_fold_matches_oracle_fold_of_oracle_series(detect, time_bin, period):
    dms = [1.0, 3.0, 6.0]
    d = Dedisperser(BW, dms, F0, 1024, 8)
    Nd = int(d.Nd.max())
    d.fold_init(period, BW, time_bin=time_bin, discard_Nd=Nd, detect=detect)
    o = O.Dedisp(BW, dms, F0, 1024, 8)
    ser = []
    for c in range(NCALLS_FOLD):
        x = noise(d.block_samples, 300 + c)
        d.filter_block(x)
        ser.append(o.filter(x.astype(np.complex128)))
    prof = d.get_profiles()
    ref = _fold_oracle(np.concatenate(ser, axis=1), period, BW, time_bin if time_bin else -1, Nd, detect)
    assert prof.shape == ref.shape
    assert d.folded_periods() > 0
    for i in range(len(dms)):
        assert rel_rms(prof[i], ref[i]) < RTOL_FOLD, (i, rel_rms(prof[i], ref[i]))


def test_fold_only_handle_equals_series_handle():
    dms = [2.0, 4.0]
    a = Dedisperser(BW, dms, F0, 1024, 8, series=False)
    b = Dedisperser(BW, dms, F0, 1024, 8, series=True)
    for d in (a, b):
        d.fold_init(0.00021, BW, time_bin=16, discard_Nd=4000)
    for c in range(6):
        x = noise(a.block_samples, 40 + c)
        a.filter_block(x)
        b.filter_block(x)
    np.testing.assert_array_equal(a.get_profiles(), b.get_profiles())
    with pytest.raises(MsosmError):
        a.get_output()


def test_fold_is_deterministic():
    res = []
    for _ in range(2):
        d = Dedisperser(BW, [1.0, 2.0, 3.0, 4.0], F0, 1024, 16, series=False)
        d.fold_init(0.00017, BW, time_bin=32, discard_Nd=2000)
        for c in range(4):
            d.filter_block(noise(d.block_samples, 7 + c))
        res.append(d.get_profiles())
    np.testing.assert_array_equal(res[0], res[1])


def test_device_tensor_input():
    torch = pytest.importorskip("torch")
    d = Dedisperser(BW, [2.0, 5.0], F0, 1024, 4)
    e = Dedisperser(BW, [2.0, 5.0], F0, 1024, 4)
    x = noise(d.block_samples, 3)
    d.filter_block(torch.from_numpy(x).cuda())
    e.filter_block(x)
    np.testing.assert_array_equal(d.get_output(), e.get_output())


def test_bad_arguments_raise():
    with pytest.raises(MsosmError):
        Dedisperser(BW, [1.0], F0, 1000, 4)  # not a power of two
    with pytest.raises(MsosmError):
        Dedisperser(BW, [-1.0], F0, 1024, 4)
    d = Dedisperser(BW, [1.0], F0, 1024, 4)
    with pytest.raises(ValueError):
        d.filter_block(noise(100, 0))
    with pytest.raises(MsosmError):
        d.fold_init(0.001, BW, time_bin=10 ** 6)


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_reset_starts_a_new_stream_like_a_fresh_handle(precision):
    # stream A for three calls, reset, stream B with a new fold period: the
    # series and profiles equal a fresh handle's on stream B
    # smears below two periods of 0.47 ms, so that the 4 calls of stream B
    # fold whole periods
    dms = [0.0, 5.0, 12.0]
    d = Dedisperser(BW, dms, F0, 4096, 6, precision=precision)
    d.fold_init(0.00031, BW, time_bin=32, discard_Nd=int(d.Nd.max()), detect="power")
    for c in range(3):
        d.filter_block(noise(d.block_samples, 100 + c))
    d.reset()
    d.fold_init(0.00047, BW, time_bin=48, discard_Nd=int(d.Nd.max()), detect="power")
    f = Dedisperser(BW, dms, F0, 4096, 6, precision=precision)
    f.fold_init(0.00047, BW, time_bin=48, discard_Nd=int(f.Nd.max()), detect="power")
    for c in range(4):
        x = noise(d.block_samples, 200 + c)
        d.filter_block(x)
        f.filter_block(x)
        np.testing.assert_array_equal(d.get_output(), f.get_output())
    np.testing.assert_array_equal(d.get_profiles(), f.get_profiles())
    assert d.folded_periods() == f.folded_periods() > 0
