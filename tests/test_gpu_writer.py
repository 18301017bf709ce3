"""The series file writer: every pushed call's series, in call order, as
get_output returns it (uint16 codec or complex64), from Python and from a
reference-style C++ driver."""
import os
import subprocess

import numpy as np
import pytest

from msosm_gpu_b200 import Dedisperser
from msosm_gpu_b200 import simulator as G
from msosm_gpu_b200.writer import SeriesWriter

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.parametrize("kind,depth,threads,precision", [("uint16", 2, 1, "fp32"), ("c64", 3, 3, "fp32"),
                                                          ("uint16", 1, 1, "fp16"), ("uint16", 4, 2, "fp16")])
def test_writer_matches_get_output(tmp_path, kind, depth, threads, precision):
    dms, count, calls = [0.0, 3.0, 7.5], 6, 7
    d = Dedisperser(16e6, dms, 1242e6, 4096, count=count, precision=precision)
    x = G.pulsar_baseband(count * 2048 * calls, 16e6, 1242e6, 5.0, 0.002, 0.05, 1.0, seed=2)
    want = []
    path = str(tmp_path / f"series_{kind}.bin")
    with SeriesWriter(d, path, kind=kind, depth=depth, threads=threads) as w:
        for c in range(calls):
            d.filter_block(x[c * count * 2048:(c + 1) * count * 2048])
            w.push()
            want.append(d.get_output(dtype=np.uint16 if kind == "uint16" else np.complex64))
    n = w.bytes_written
    got = np.fromfile(path, np.uint16 if kind == "uint16" else np.complex64)
    assert n == got.nbytes
    want = np.concatenate([a.reshape(-1) for a in want])
    np.testing.assert_array_equal(got, want)
    d.close()


def test_writer_rejects_fold_only_handles(tmp_path):
    from msosm_gpu_b200._abi import MsosmError
    d = Dedisperser(16e6, [1.0], 1242e6, 4096, count=2, series=False)
    with pytest.raises(MsosmError):
        SeriesWriter(d, str(tmp_path / "x.bin"))
    d.close()


def test_cpp_writer_driver(tmp_path):
    exe = str(tmp_path / "writer_demo")
    libdir = os.path.join(ROOT, "msosm_gpu_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(HERE, "cpp", "writer_demo.cpp"), "-L", libdir, "-lmsosm_b200",
                    f"-Wl,-rpath,{libdir}"], check=True, capture_output=True, text=True)
    out = str(tmp_path / "w.bin")
    numDMs, count, calls = 4, 3, 5
    r = subprocess.run([exe, str(numDMs), str(count), str(calls), out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.uint16).reshape(calls, numDMs, count * 2048, 2)
    sim = G.SimulatedComplexSignal(16e6, 12.0, 1242e6, 0.0005, "uint16", seed=17)
    process_len = count * 2048
    sim.generate_pulsar_signal(process_len * calls // sim.Np + 1, True, -3.0)
    dms = [1.0 + 0.5 * i for i in range(numDMs)]
    d = Dedisperser(16e6, dms, 1242e6, 4096, count=count)
    for c in range(calls):
        d.filter_block(sim.signal_u16[c * process_len:(c + 1) * process_len])
        np.testing.assert_array_equal(got[c], d.get_output(dtype=np.uint16))
    assert f"bytes {got.nbytes}" in r.stdout
    d.close()
