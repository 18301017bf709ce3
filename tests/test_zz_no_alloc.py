"""The allocation-free filter-design entry point, through the C ABI.

Callers that cannot call cudaMalloc (pipelines that reserve all device
memory before an observation, hosts whose allocator owns the device, code
that redesigns a filter mid-pass) use msosm_prepare_dedisp_params_noalloc:
the output is their own device buffer and the scratch is a fixed array
inside the library.  Its result must equal the allocating entry point's
(msosm_prepare_dedisp_params) within the tolerance of the other GPU tests,
on two calls in a row (the second call reuses the scratch the first left
behind).  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from msosm_gpu_b200 import _abi, prepare

pytestmark = pytest.mark.gpu

RTOL = 2e-5


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def test_noalloc_design_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    L = _abi.lib()
    cases = [(16e6, 73.2, 1242e6, 2048), (64e6, 37.5, 1368e6, 4096)]
    for bw, dm, f0, M in cases:
        ref = prepare.dedisp_params(bw, dm, f0, M)
        out = torch.full((2 * M,), complex(7.0, 7.0), dtype=torch.complex64, device="cuda")
        torch.cuda.synchronize()
        st = L.msosm_prepare_dedisp_params_noalloc(bw, dm, f0, M, ctypes.c_void_p(out.data_ptr()), None)
        assert st == _abi.OK, L.msosm_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_rms(got, ref) < RTOL, rel_rms(got, ref)


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
