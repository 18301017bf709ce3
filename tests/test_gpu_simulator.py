"""The device simulator against its CPU restatement (oracle/sim_ref.py) and
the reference simulator's own output (tests/golden): the counter-based
normals bit for bit, AWGN, the reference's two-spike SimulatedComplexSignal,
the streaming dispersed pulsar against an FP64 overlap-save with the
reference's dispersion filter, chunking invariance, and a dedispersion
round trip."""
import math

import numpy as np
import pytest

import oracle as O
import sim_ref as R
from msosm_gpu_b200 import Dedisperser
from msosm_gpu_b200 import simulator as G

pytestmark = pytest.mark.gpu

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
META = json.load(open(os.path.join(HERE, "golden", "reference_host.json")))
ARR = np.load(os.path.join(HERE, "golden", "reference_host.npz"))


def ulp_diff(a, b):
    a = np.ascontiguousarray(a, np.complex64).view(np.float32)
    b = np.ascontiguousarray(b, np.complex64).view(np.float32)
    ia, ib = a.view(np.int32).astype(np.int64), b.view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


@pytest.mark.parametrize("seed,start,tag", [(0, 0, 0), (123456789012345, (1 << 32) - 5000, 1), (7, 3, 0)])
def test_normals_match_cpu(seed, start, tag):
    n = 1 << 18
    g1, g2 = G.normals(seed, start, n, tag)
    c1, c2 = R.normals(seed, start, n, tag)
    for g, c in ((g1, c1), (g2, c2)):
        d = ulp_diff(g, c)
        # Box-Muller in double rounded once to float: equal except where the
        # device and host libm differ by an ulp right at a rounding boundary
        assert d.max() <= 1
        assert np.count_nonzero(d) <= 4, np.count_nonzero(d)


def test_awgn_modes():
    n = 1 << 16
    a = G.AWGN(12.0, n, seed=5).generateNoiseSamples()
    z, _ = R.normals(5, 0, n, R.TAG_AWGN)
    sigma = np.float32(math.sqrt(10.0 ** float(np.float32(-12.0) / np.float32(10))))
    want = (z.astype(np.complex128) * (float(sigma) / math.sqrt(2.0))).astype(np.complex64)
    assert ulp_diff(a, want).max() <= 1
    b = G.AWGN(0.5, 2.0, n, seed=5).generateNoiseSamples()
    wr = (z.real * np.float32(2.0) + np.float32(0.5)).astype(np.float32)
    assert ulp_diff(b.real + 0j, wr + 0j).max() <= 1
    assert abs(b.real.mean() - 0.5) < 0.05 and abs(b.real.std() - 2.0) < 0.05


def test_two_spike_matches_reference_simulator():
    s = META["simulate"]
    sim = G.SimulatedComplexSignal(s["bw"], s["dm"], s["f0"], s["period"], "uint16")
    sim.generate_pulsar_signal(s["repeat"], False, 0.0)
    ref = ARR["simulate_signal"].view(np.complex64)
    assert sim.signal_size == ref.size == s["Np"] * s["repeat"]
    assert np.abs(sim.signal - ref).max() / np.abs(ref).max() < 1e-5
    # the codec bit for bit on the device's own values; decoded, within one
    # count of the reference's.  Where the exact convolution is 0 (after the
    # last delta of a period when the smear is shorter than a period) the
    # device has 0 -- the blank code -- and the reference's FFT round-off
    # (~1e-9) codes as 32768 or 32767: both decode to 0 or -1.
    np.testing.assert_array_equal(sim.signal_u16, R.quantise_reference(sim.signal))
    ur = ARR["simulate_signal_u16"].reshape(-1, 2).astype(np.int64)
    ud = sim.signal_u16.astype(np.int64)
    dec = lambda u: np.where(u == 0, 0, u - 32768)  # noqa: E731 (gpu_kernel.cu:276-299)
    assert np.abs(dec(ud) - dec(ur)).max() <= 1
    exact_zero = (sim.signal.real == 0) & (sim.signal.imag == 0)
    assert np.all(np.abs(ref[exact_zero]) < 1e-6)
    # and the FP64 oracle
    x = O.simulate_two_spike(s["bw"], s["dm"], s["f0"], s["period"], s["repeat"])
    assert np.abs(sim.signal - x).max() / np.abs(x).max() < 1e-5


@pytest.mark.parametrize("dm,period", [(75.0, 0.005), (30.0, 0.0011)])
def test_two_spike_long_smear_against_oracle(dm, period):
    sim = G.SimulatedComplexSignal(16e6, dm, 1242e6, period)
    sim.generate_pulsar_signal(2, False, 0.0)
    x = O.simulate_two_spike(16e6, dm, 1242e6, period, 2)
    assert sim.range == -(-sim.Nd // sim.Np)
    assert np.abs(sim.signal - x).max() / np.abs(x).max() < 2e-5


def test_two_spike_noise():
    s = META["simulate"]
    clean = G.SimulatedComplexSignal(s["bw"], s["dm"], s["f0"], s["period"], "uint16", seed=9)
    clean.generate_pulsar_signal(4, False, 0.0)
    noisy = G.SimulatedComplexSignal(s["bw"], s["dm"], s["f0"], s["period"], "uint16", seed=9)
    noisy.generate_pulsar_signal(4, True, -10.0)
    assert noisy.signal_power == clean.signal_power
    sigma = np.float32(math.sqrt(10.0 ** float(np.float32(-(np.float32(-10.0) - np.float32(clean.signal_power)))
                                              / np.float32(10))))
    z, _ = R.normals(9, 0, noisy.signal_size, R.TAG_AWGN)
    noise = (z.astype(np.complex128) * (float(sigma) / math.sqrt(2.0))).astype(np.complex64)
    want = np.empty_like(noise)
    want.real = clean.signal.real + noise.real
    want.imag = clean.signal.imag + noise.imag
    assert ulp_diff(noisy.signal, want).max() <= 1
    np.testing.assert_array_equal(noisy.signal_u16, R.quantise_reference(noisy.signal))
    # 10 dB more noise than signal power
    p = np.mean(np.abs(noisy.signal - clean.signal) ** 2)
    assert abs(10 * np.log10(p) - (clean.signal_power + 10.0)) < 0.1


def osm_reference(bw, f0, dm, period, fwhm, snr, seed, n, M):
    H = O.dedisp_params(bw, dm, f0, M, +1)
    return R.pulsar(H, M, seed, n, bw, period, fwhm, 0.5, snr)


@pytest.mark.parametrize("dm", [0.0, 5.0, 20.0])
def test_pulsar_matches_fp64_restatement(dm):
    bw, f0, period, fwhm, snr, seed = 16e6, 1242e6, 0.0031, 0.05, 2.0, 4
    sim = G.PulsarSimulator(bw, f0, dm, period, fwhm, snr, seed=seed, min_chunk=1 << 17)
    n = 2 * sim.chunk
    x = np.concatenate([sim.next()[0], sim.next()[0]])
    assert sim.next_sample == n
    ref = osm_reference(bw, f0, dm, period, fwhm, snr, seed, n, sim.M) if sim.M else \
        R.pulsar(None, 0, seed, n, bw, period, fwhm, 0.5, snr)
    err = np.sqrt(np.mean(np.abs(x - ref) ** 2) / np.mean(np.abs(ref) ** 2))
    assert err < (1e-7 if dm == 0 else 3e-6), err


def test_pulsar_chunking_invariant():
    kw = dict(bw=16e6, f0=1242e6, dm=12.0, period=0.002, fwhm=0.04, snr=1.0, seed=3)
    a = G.PulsarSimulator(**kw, min_chunk=1)
    b = G.PulsarSimulator(**kw, min_chunk=4 * a.M)
    xa = np.concatenate([a.next()[0] for _ in range(4)])
    xb, ub = b.next(u16_scale=1000.0)
    np.testing.assert_array_equal(xa, xb)
    q = np.stack([np.rint(xb.real.astype(np.float64) * 1000.0), np.rint(xb.imag.astype(np.float64) * 1000.0)], 1)
    np.testing.assert_array_equal(ub, np.clip(q + 32768, 1, 65535).astype(np.uint16))


def test_pulsar_on_device_and_dedispersed():
    torch = pytest.importorskip("torch")
    bw, f0, dm, period = 16e6, 1242e6, 30.0, 0.0025
    n = 1 << 22
    xd = G.pulsar_baseband(n, bw, f0, dm, period, 0.03, 0.5, seed=1, device=torch.device("cuda"))
    xh = G.pulsar_baseband(n, bw, f0, dm, period, 0.03, 0.5, seed=1)
    np.testing.assert_array_equal(xd.cpu().numpy(), xh)
    dms = [0.0, 15.0, 29.0, 30.0, 31.0, 45.0]
    d = Dedisperser(bw, dms, f0, 4096, count=n // 2048, series=False)
    d.fold_init(period, bw, time_bin=256, discard_Nd=int(d.Nd.max()), detect="power")
    d.filter_block(xd)
    prof = d.get_profiles()
    snr = (prof.max(1) - np.median(prof, 1)) / prof.std(1)
    assert int(np.argmax(snr)) == dms.index(30.0)


def test_cpp_dropin_classes(tmp_path):
    import subprocess
    root = os.path.dirname(HERE)
    libdir = os.path.join(root, "msosm_gpu_b200")
    exe = str(tmp_path / "simulate_demo")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(root, "include"), "-o", exe,
                    os.path.join(HERE, "cpp", "simulate_demo.cpp"), "-L", libdir, "-lmsosm_b200",
                    f"-Wl,-rpath,{libdir}"], check=True, capture_output=True, text=True)
    out = str(tmp_path / "sim.bin")
    args = (16e6, 5.0, 1242e6, 0.0005, 3, 1, -5.0, 42, 5000)
    r = subprocess.run([exe, *[repr(a) for a in args], out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    sim = G.SimulatedComplexSignal(16e6, 5.0, 1242e6, 0.0005, "uint16", seed=42)
    sim.generate_pulsar_signal(3, True, -5.0)
    n = sim.signal_size
    raw = open(out, "rb").read()
    sig = np.frombuffer(raw[:8 * n], np.complex64)
    u16 = np.frombuffer(raw[8 * n:12 * n], np.uint16).reshape(-1, 2)
    noise = np.frombuffer(raw[12 * n:], np.complex64)
    np.testing.assert_array_equal(sig, sim.signal)
    np.testing.assert_array_equal(u16, sim.signal_u16)
    np.testing.assert_array_equal(noise, G.AWGN(-5.0, 5000, seed=42).generateNoiseSamples())
    assert f"Np {sim.Np} Nd {sim.Nd}" in r.stdout
