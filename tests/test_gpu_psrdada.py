"""The two-polarisation PSRDADA pipeline end to end (msosm_psrdada.cpp:92-144):
a simulated two-pol pulsar written as a PSRDADA file, read, dedispersed per
polarisation, sqrt(|a|^2 + |b|^2) detected and folded on the device, against
the FP64 oracle running the same steps on the same file."""
import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import psrdada as P
from msosm_gpu_b200 import simulate as S

pytestmark = pytest.mark.gpu

BW_MHZ, FREQ_MHZ = 16.0, 1250.0


def oracle_fold(path, dm, period, fftpoint, time_bin):
    f = P.PSRDADA(path)
    bw = np.float32(f.bw)
    f0 = np.float32(np.float32(f.fc) - bw / np.float32(2))
    bw = float(np.float32(bw * np.float32(1e6)))
    f0 = float(np.float32(f0 * np.float32(1e6)))
    oa, ob = O.Dedisp(bw, [dm], f0, fftpoint, 1), O.Dedisp(bw, [dm], f0, fftpoint, 1)
    f.initBuffer(oa.M)
    fold = O.Fold(period, bw, oa.M, time_bin)
    fold.discard_samples(int(oa.Nd[0]))
    first = True
    for _ in range(f.readCount):
        f.readSamples()
        if first:
            if f.pol1_in[0, 0] == 0:
                continue
            first = False
        ya = oa.filter(O.decode_uint16(f.pol1_in))[0]
        yb = ob.filter(O.decode_uint16(f.pol2_in))[0]
        fold.fold_data(O.intensity(ya, yb))
    return fold.fold_data_bins()


@pytest.mark.parametrize("blank_reads", [0, 2])
def test_psrdada_two_pol_fold_matches_oracle(tmp_path, blank_reads):
    dm, period, fftpoint, tb = 5.0, 0.0011, 8192, 64
    bw, f0 = BW_MHZ * 1e6, (FREQ_MHZ - BW_MHZ / 2) * 1e6
    n = 4096 * 40
    xa = S.pulsar_baseband(n, bw, f0, dm, period, 0.05, 3.0, seed=3)
    xb = S.pulsar_baseband(n, bw, f0, dm, period, 0.05, 3.0, seed=4)
    a, b = S.quantise_uint16(xa, 300.0), S.quantise_uint16(xb, 300.0)
    # blank data at the head of the file (the pipeline skips those reads)
    a[:blank_reads * 4096] = 0
    b[:blank_reads * 4096] = 0
    path = str(tmp_path / "sim.dada")
    P.write_dada(path, a, b, BW_MHZ, FREQ_MHZ)
    ours = P.fold_file(path, dm, period, fftpoint=fftpoint, time_bin=tb)
    ref = oracle_fold(path, dm, period, fftpoint, tb)
    assert ours.shape == (tb,) and np.any(ours)
    err = float(np.sqrt(np.mean((ours - ref) ** 2) / np.mean(ref ** 2)))
    assert err < 2e-5, err
    written = np.loadtxt(str(tmp_path / "sim_dedisp_folded.txt"))
    np.testing.assert_allclose(written, ours, rtol=1e-5)
    # the pulse is found at the injected phase: profile peak well above the median
    assert ours.max() > 1.5 * np.median(ours)
    # reading on a second thread into pinned buffers changes nothing
    st = {}
    same = P.fold_file(path, dm, period, fftpoint=fftpoint, time_bin=tb, write=False, overlap=False, stats=st)
    np.testing.assert_array_equal(same, ours)
    assert st["reads"] == 40 and st["samples"] == 40 * 4096


@pytest.mark.parametrize("fftpoint", [4096, 16384])
def test_psrdada_two_pol_fold_on_tensor_cores(tmp_path, fftpoint):
    # the same pipeline with both polarisations' inverse transforms on the
    # tensor cores (f16 operands): the folded two-pol amplitude profile
    # within the tensor path's profile bound (1e-4) of the FP64 oracle
    dm, period, tb = 5.0, 0.0011, 64
    bw, f0 = BW_MHZ * 1e6, (FREQ_MHZ - BW_MHZ / 2) * 1e6
    n = 8192 * 20
    xa = S.pulsar_baseband(n, bw, f0, dm, period, 0.05, 3.0, seed=5)
    xb = S.pulsar_baseband(n, bw, f0, dm, period, 0.05, 3.0, seed=6)
    path = str(tmp_path / "tc.dada")
    P.write_dada(path, S.quantise_uint16(xa, 300.0), S.quantise_uint16(xb, 300.0), BW_MHZ, FREQ_MHZ)
    ours = P.fold_file(path, dm, period, fftpoint=fftpoint, time_bin=tb, precision="fp16", write=False)
    ref = oracle_fold(path, dm, period, fftpoint, tb)
    assert ours.shape == (tb,) and np.any(ours)
    err = float(np.sqrt(np.mean((ours - ref) ** 2) / np.mean(ref ** 2)))
    assert err < 1e-4, err


def test_psrdada_streaming_reads(tmp_path):
    """Many reads with count > 1 (several FFT blocks per read): the
    overlapped reader keeps order and covers the whole file."""
    dm, period, fftpoint, tb, count = 8.0, 0.0021, 4096, 128, 4
    bw, f0 = BW_MHZ * 1e6, (FREQ_MHZ - BW_MHZ / 2) * 1e6
    n = 2048 * count * 25
    a = S.quantise_uint16(S.pulsar_baseband(n, bw, f0, dm, period, 0.04, 2.0, seed=8), 300.0)
    b = S.quantise_uint16(S.pulsar_baseband(n, bw, f0, dm, period, 0.04, 2.0, seed=9), 300.0)
    path = str(tmp_path / "stream.dada")
    P.write_dada(path, a, b, BW_MHZ, FREQ_MHZ)
    st = {}
    ov = P.fold_file(path, dm, period, fftpoint=fftpoint, count=count, time_bin=tb, write=False, stats=st)
    sq = P.fold_file(path, dm, period, fftpoint=fftpoint, count=count, time_bin=tb, write=False, overlap=False)
    np.testing.assert_array_equal(ov, sq)
    assert st["reads"] == 25 and st["samples"] == n


def test_psrdada_cpp_driver_matches_python_pipeline(tmp_path):
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "msosm_gpu_b200")
    exe = str(tmp_path / "psrdada_demo")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(root, "include"), "-o", exe,
                    os.path.join(root, "tests", "cpp", "psrdada_demo.cpp"), "-L", libdir, "-lmsosm_b200",
                    f"-Wl,-rpath,{libdir}"], check=True, capture_output=True, text=True)
    dm, period, fftpoint, tb = 20.0, 0.0031, 16384, 128
    bw, f0 = BW_MHZ * 1e6, (FREQ_MHZ - BW_MHZ / 2) * 1e6
    n = 8192 * 24
    a = S.quantise_uint16(S.pulsar_baseband(n, bw, f0, dm, period, 0.03, 2.0, seed=5), 300.0)
    b = S.quantise_uint16(S.pulsar_baseband(n, bw, f0, dm, period, 0.03, 2.0, seed=6), 300.0)
    path = str(tmp_path / "cpp.dada")
    P.write_dada(path, a, b, BW_MHZ, FREQ_MHZ)
    r = subprocess.run([exe, path, str(dm), str(period), str(fftpoint), str(tb)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    cpp = np.loadtxt(str(tmp_path / "cpp_dedisp_folded.txt"))
    py = P.fold_file(path, dm, period, fftpoint=fftpoint, time_bin=tb, write=False)
    np.testing.assert_allclose(cpp, py, rtol=1e-5)
