"""The simulator's CPU side: the Philox4x32-10 restatement of the checker
against the generator's published known-answer vectors, the reference's
uint16 codec restated against the reference simulator's own output, and the
host-side sizes and argument checks of the C ABI (no GPU needed)."""
import ctypes
import json
import os

import numpy as np
import pytest

import sim_ref as R
from msosm_gpu_b200 import _abi
from msosm_gpu_b200._abi import MsosmError, check, lib

HERE = os.path.dirname(os.path.abspath(__file__))
META = json.load(open(os.path.join(HERE, "golden", "reference_host.json")))
ARR = np.load(os.path.join(HERE, "golden", "reference_host.npz"))

# Philox4x32-10 known-answer vectors of the generator's authors (counter,
# key, output), Salmon et al., SC11 2011
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(ctr, key, want):
    out = R.philox4x32_10(np.array([ctr], np.uint32), key)[0]
    assert tuple(int(v) for v in out) == want


def test_normals_are_unit_and_independent():
    z1, z2 = R.normals(11, (1 << 32) - 4096, 1 << 18)
    for z in (z1, z2):
        for c in (z.real, z.imag):
            assert abs(c.mean()) < 0.01 and abs(c.var() - 1) < 0.01
    assert abs(np.mean(z1.real * z2.real)) < 0.01
    # sample i depends on (seed, i, tag) only
    a1, _ = R.normals(11, (1 << 32) - 4096 + 100, 50)
    np.testing.assert_array_equal(a1, z1[100:150])


def test_reference_codec_restated():
    s = META["simulate"]
    sig = ARR["simulate_signal"].view(np.complex64)
    u = R.quantise_reference(sig)
    np.testing.assert_array_equal(u.reshape(-1), ARR["simulate_signal_u16"])


def test_two_spike_shape_matches_reference():
    s = META["simulate"]
    info = _abi.SimTwoSpikeInfo()
    check(lib().msosm_sim_two_spike_shape(s["bw"], s["dm"], s["f0"], s["period"], ctypes.byref(info)))
    assert info.Np == s["Np"] and info.Nd == s["Nd"]
    assert info.range == 1 and info.order == 8192
    check(lib().msosm_sim_two_spike_shape(16e6, 75.0, 1242e6, 0.005, ctypes.byref(info)))
    assert info.Np == 80000 and info.range == -(-info.Nd // info.Np) and info.order == 1 << 18


@pytest.mark.parametrize("args", [(16e6, 5.0, 1242e6, 0.0), (16e6, -1.0, 1242e6, 0.001),
                                  (0.0, 5.0, 1242e6, 0.001), (16e6, 5.0, 1242e6, 1e-7)])
def test_two_spike_rejects_bad_parameters(args):
    info = _abi.SimTwoSpikeInfo()
    assert lib().msosm_sim_two_spike_shape(*args, ctypes.byref(info)) == _abi.ERR_BAD_ARG


@pytest.mark.parametrize("field,value", [("bw", 0.0), ("dm", -1.0), ("period", 0.0), ("fwhm", 0.0),
                                         ("snr", -0.1)])
def test_pulsar_rejects_bad_parameters(field, value):
    p = _abi.SimPulsarParams(bw=16e6, f0=1242e6, dm=5.0, period=0.003, fwhm=0.03, centre=0.5, snr=0.1, seed=0)
    setattr(p, field, value)
    h = ctypes.c_void_p()
    assert lib().msosm_sim_pulsar_create(ctypes.byref(p), 0, ctypes.byref(h)) == _abi.ERR_BAD_ARG
    assert not h.value


def test_disperse_needs_osm():
    bw, dm, f0 = (ctypes.c_float * 1)(16e6), (ctypes.c_float * 1)(5.0), (ctypes.c_float * 1)(1242e6)
    h = ctypes.c_void_p()
    st = lib().msosm_dedisp_create(bw, dm, f0, 1, 0, 1, 0, _abi.FLAG_DISPERSE, ctypes.byref(h))
    assert st == _abi.ERR_BAD_ARG
    with pytest.raises(MsosmError):
        check(st)


def test_host_buffers():
    p = ctypes.c_void_p()
    check(lib().msosm_host_alloc(1024, 0, ctypes.byref(p)))
    assert p.value
    ctypes.memset(p, 7, 1024)
    check(lib().msosm_host_free(p, 0))


def test_cpp_dropin_compiles(tmp_path):
    import subprocess
    root = os.path.dirname(HERE)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(root, "include"), "-o",
                    str(tmp_path / "simulate_demo"), os.path.join(HERE, "cpp", "simulate_demo.cpp"),
                    "-L", os.path.join(root, "msosm_gpu_b200"), "-lmsosm_b200"], check=True, capture_output=True,
                   text=True)


def test_writer_host_checks(tmp_path):
    w = ctypes.c_void_p()
    assert lib().msosm_writer_create(None, str(tmp_path / "x").encode(), 0, 2, 1, ctypes.byref(w)) == _abi.ERR_BAD_ARG
    assert lib().msosm_writer_close(None, None) == _abi.OK
    subprocess_compile(tmp_path, "writer_demo")


def subprocess_compile(tmp_path, name):
    import subprocess
    root = os.path.dirname(HERE)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(root, "include"), "-o",
                    str(tmp_path / name), os.path.join(HERE, "cpp", name + ".cpp"),
                    "-L", os.path.join(root, "msosm_gpu_b200"), "-lmsosm_b200"], check=True, capture_output=True,
                   text=True)
