"""The allocation-free filter-design entry point, through the C ABI.

Some callers of this library cannot call cudaMalloc: a pipeline that
reserves all of its device memory before an observation starts and may not
allocate while samples stream in, a host framework whose own allocator owns
the device, code that redesigns one trial's filter in the middle of a pass
without the device-wide synchronisation an allocation brings.  They use
msosm_prepare_dedisp_params_noalloc: the output is their own device buffer
and the design's scratch is a fixed array inside the library (M <= 8192).

Its result must equal the allocating entry point's (msosm_prepare_dedisp_params)
within the tolerance of the other GPU tests, call after call: every case runs
two calls in a row, the second reusing the scratch the first left behind.
It is also held to the filters the reference's own host code designed
(tests/golden) and, at sizes the fixtures lack (M = 32 and the maximum
M = 8192), to the FP64 oracle.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import _abi, prepare

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
RTOL = 2e-5


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def design(torch, bw, dm, f0, M, stream=None):
    """One call of the allocation-free entry into a fresh device buffer."""
    L = _abi.lib()
    out = torch.full((2 * M,), complex(7.0, 7.0), dtype=torch.complex64, device="cuda")
    torch.cuda.synchronize()
    handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    st = L.msosm_prepare_dedisp_params_noalloc(bw, dm, f0, M, ctypes.c_void_p(out.data_ptr()), handle)
    assert st == _abi.OK, L.msosm_last_error()
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_design_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    cases = [(16e6, 73.2, 1242e6, 2048), (64e6, 37.5, 1368e6, 4096),
             (16e6, 0.8, 1242e6, 32), (64e6, 150.0, 1368e6, 8192)]
    for bw, dm, f0, M in cases:
        ref = prepare.dedisp_params(bw, dm, f0, M)
        for _ in range(2):
            got = design(torch, bw, dm, f0, M)
            assert rel_rms(got, ref) < RTOL, (M, rel_rms(got, ref))


def test_noalloc_same_size_different_trials_in_a_row():
    # two calls of one size with different DMs: the second must match its own
    # reference, not anything the first left in the scratch
    torch = pytest.importorskip("torch")
    for M in (4096, 8192):
        for dm in (25.0, 180.0):
            got = design(torch, 64e6, dm, 1368e6, M)
            assert rel_rms(got, prepare.dedisp_params(64e6, dm, 1368e6, M)) < RTOL, (M, dm)


def test_noalloc_matches_reference_golden_and_oracle():
    torch = pytest.importorskip("torch")
    meta = json.load(open(os.path.join(HERE, "golden", "reference_host.json")))
    arr = np.load(os.path.join(HERE, "golden", "reference_host.npz"))
    checked = 0
    for k, s in enumerate(meta["msosm"]):
        if s["M"] < 32 or s["M"] > 8192:
            continue
        Hr = arr[f"msosm{k}_H"].astype(np.float64).view(np.complex128)
        got = design(torch, s["bw"], s["dm"], s["f0"], s["M"])
        assert rel_rms(got, Hr) < RTOL, (k, rel_rms(got, Hr))
        checked += 1
    assert checked >= 5
    for bw, dm, f0, M in [(16e6, 0.8, 1242e6, 32), (64e6, 150.0, 1368e6, 8192)]:
        got = design(torch, bw, dm, f0, M)
        assert rel_rms(got, O.dedisp_params(bw, dm, f0, M)) < RTOL, M


def test_noalloc_on_a_caller_stream():
    torch = pytest.importorskip("torch")
    s = torch.cuda.Stream()
    for dm in (50.0, 73.2):
        got = design(torch, 16e6, dm, 1242e6, 2048, stream=s)
        assert rel_rms(got, prepare.dedisp_params(16e6, dm, 1242e6, 2048)) < RTOL


def test_noalloc_rejects_sizes_beyond_its_maximum():
    torch = pytest.importorskip("torch")
    L = _abi.lib()
    out = torch.zeros(2 * 16384, dtype=torch.complex64, device="cuda")
    st = L.msosm_prepare_dedisp_params_noalloc(16e6, 1.0, 1242e6, 16384, ctypes.c_void_p(out.data_ptr()), None)
    assert st == _abi.ERR_BAD_ARG
    assert b"8192" in L.msosm_last_error()
    host = np.zeros(2 * 1024, np.complex64)
    st = L.msosm_prepare_dedisp_params_noalloc(16e6, 1.0, 1242e6, 1024, ctypes.c_void_p(host.ctypes.data), None)
    assert st == _abi.ERR_BAD_ARG
    st = L.msosm_prepare_dedisp_params_noalloc(16e6, -1.0, 1242e6, 1024, ctypes.c_void_p(out.data_ptr()), None)
    assert st == _abi.ERR_BAD_ARG


def test_noalloc_rejects_memory_of_another_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    L = _abi.lib()
    other = torch.zeros(2 * 1024, dtype=torch.complex64, device="cuda:1")
    torch.cuda.set_device(0)
    st = L.msosm_prepare_dedisp_params_noalloc(16e6, 1.0, 1242e6, 1024, ctypes.c_void_p(other.data_ptr()), None)
    assert st == _abi.ERR_BAD_ARG
    assert b"device" in L.msosm_last_error()
