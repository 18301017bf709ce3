"""The C++ drop-in header (include/msosm_gpu_b200.hpp): a reference-style
driver compiled with g++ against it, run on the GPU, must produce what the
same library gives through the Python binding, and the single-DM / stream /
loop classes must agree with the DM-concurrent one."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from msosm_gpu_b200 import Dedisperser

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_demo.cpp")
LIBDIR = os.path.join(ROOT, "msosm_gpu_b200")


def compile_demo(out):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", out, SRC,
           "-L", LIBDIR, "-lmsosm_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_dropin_header_compiles():
    with tempfile.TemporaryDirectory() as td:
        compile_demo(os.path.join(td, "demo"))


@pytest.mark.gpu
def test_dropin_classes_match_python_binding():
    calls, count, M = 4, 4, 512
    blk = count * M
    rng = np.random.default_rng(21)
    x = np.clip(np.rint(rng.standard_normal((blk * calls, 2)) * 1000) + 32768, 1, 65535).astype(np.uint16)
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "demo")
        compile_demo(exe)
        fin, fout = os.path.join(td, "in.u16"), os.path.join(td, "out.c64")
        x.tofile(fin)
        r = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        y = np.fromfile(fout, np.complex64)
    dms = [1.0, 3.5, 7.0]
    off = 0

    def take(n):
        nonlocal off
        v = y[off:off + n]
        off += n
        return v

    conc = np.stack([take(3 * blk).reshape(3, blk) for _ in range(calls)], 1).reshape(3, -1)
    single = np.concatenate([take(blk) for _ in range(calls)])
    osm = np.concatenate([take(blk) for _ in range(calls)])
    streams = [[], []]
    for _ in range(calls):
        streams[0].append(take(blk))
        streams[1].append(take(blk))
    loop = [[], [], []]
    for _ in range(calls):
        for i in range(3):
            loop[i].append(take(blk))
    assert off == y.size

    def py(dm_list, osm_mode=False):
        d = Dedisperser(16e6, dm_list, 1242e6, 1024, count, osm=osm_mode)
        res = []
        for c in range(calls):
            d.filter_block(x[c * blk:(c + 1) * blk])
            res.append(d.get_output())
        return np.concatenate(res, 1)

    np.testing.assert_array_equal(conc, py(dms))
    np.testing.assert_array_equal(single, py([3.5])[0])
    np.testing.assert_array_equal(osm, py([0.1], True)[0])
    np.testing.assert_array_equal(np.concatenate(streams[0]), py([1.0])[0])
    np.testing.assert_array_equal(np.concatenate(streams[1]), py([3.5])[0])
    for i in range(3):
        np.testing.assert_array_equal(np.concatenate(loop[i]), conc[i])


@pytest.mark.gpu
@pytest.mark.parametrize("fftpoint", [4096, 8192, 16384])
def test_dropin_classes_on_tensor_cores(fftpoint):
    # use_tensor_cores(true) before the reference's classes are initialised:
    # the driver's series equal the Python binding's f16 path bit for bit
    # and match the FP64 oracle within the tensor path's series bound
    import oracle as O
    calls, count = 3, 2
    blk = count * fftpoint // 2
    rng = np.random.default_rng(22)
    x = np.clip(np.rint(rng.standard_normal((blk * calls, 2)) * 1000) + 32768, 1, 65535).astype(np.uint16)
    src = os.path.join(ROOT, "tests", "cpp", "dropin_tensor_demo.cpp")
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "demo")
        subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", exe, src,
                        "-L", LIBDIR, "-lmsosm_b200", f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True,
                       text=True)
        fin, fout = os.path.join(td, "in.u16"), os.path.join(td, "out.c64")
        x.tofile(fin)
        r = subprocess.run([exe, str(fftpoint), fin, fout], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (r.returncode, r.stderr)
        y = np.fromfile(fout, np.complex64).reshape(calls, 4 * blk)
    conc = np.concatenate([y[c, :3 * blk].reshape(3, blk) for c in range(calls)], 1)
    single = np.concatenate([y[c, 3 * blk:] for c in range(calls)])
    dms = [0.5, 20.0, 60.0]
    d = Dedisperser(16e6, dms, 1242e6, fftpoint, count, precision="fp16")
    o = O.Dedisp(16e6, dms, 1242e6, fftpoint, count)
    py, ref = [], []
    for c in range(calls):
        blk_in = x[c * blk:(c + 1) * blk]
        d.filter_block(blk_in)
        py.append(d.get_output())
        ref.append(o.filter(O.decode_uint16(blk_in)))
    py, ref = np.concatenate(py, 1), np.concatenate(ref, 1)
    np.testing.assert_array_equal(conc, py)
    np.testing.assert_array_equal(single, py[1])
    for i in range(3):
        e = float(np.sqrt(np.mean(np.abs(conc[i] - ref[i]) ** 2) / np.mean(np.abs(ref[i]) ** 2)))
        assert e < 1.5e-3, (dms[i], e)


@pytest.mark.gpu
def test_fold_raw_state_and_per_trial_prepare_fields():
    import oracle as O
    src = os.path.join(ROOT, "tests", "cpp", "fold_state_demo.cpp")
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "fold_state")
        subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", exe, src,
                        "-L", LIBDIR, "-lmsosm_b200", f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = {l.split()[0]: l.split()[1:] for l in r.stdout.splitlines()}
    ps = int(lines["period_samples"][0])
    assert ps == 100
    # 640 samples: periods 0..5 complete, 40 samples of period 6 in progress
    t = np.arange(640)
    val = np.where(t % 7 == 0, 0.0, 1.0 + t)
    want_count = [(val[:600].reshape(6, 100)[:, p] != 0).sum() for p in range(100)]
    assert [int(v) for v in lines["fold_count"]] == want_count
    assert [float(v) for v in lines["tmp_fold"]] == list(val[600:640])
    mins = [O.msosm_min_order(O.nd(16e6, dm, 1242e6)) for dm in (10.0, 50.0, 73.2)]
    assert [int(v) for v in lines["M_min"][:3]] == mins and int(lines["M_min"][4]) == max(mins)
    prep, hand = lines["prepared"], lines["handle"]
    for dm_i, dm in enumerate((10.0, 50.0, 73.2)):
        dc, dp = O.segmentation(16e6, dm, 1242e6, 2048)
        assert int(prep[1 + dm_i]) == dc and int(hand[1 + dm_i]) == dc
    assert int(prep[5]) == O.segmentation(16e6, 73.2, 1242e6, 2048)[1][100] == int(hand[5])
    H = O.dedisp_params(16e6, 73.2, 1242e6, 2048)
    for v in (prep, hand):
        assert abs(complex(float(v[7]), float(v[8])) - H[7]) < 2e-5 * np.abs(H).max()
    assert [int(v) for v in hand[10:13]] == mins and int(hand[14]) == O.nd(16e6, 73.2, 1242e6)
