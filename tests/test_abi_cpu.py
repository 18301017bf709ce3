"""The C ABI on a machine without a GPU: the library loads, exports every
symbol include/msosm_b200.h declares, and its host-side arithmetic (filter
parameters, segmentation, fold planner) equals the reference's (golden
fixtures) and the oracle's."""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import cuda_available
from msosm_gpu_b200 import _abi, prepare

HERE = os.path.dirname(os.path.abspath(__file__))
META = json.load(open(os.path.join(HERE, "golden", "reference_host.json")))
ARR = np.load(os.path.join(HERE, "golden", "reference_host.npz"))


def test_library_exports_every_header_symbol():
    L = _abi.lib()
    names = _abi.header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_error_string():
    assert _abi.lib().msosm_version() >= 100
    st = _abi.lib().msosm_prepare_nd(-1.0, 1.0, 1.0, None)
    assert st == _abi.ERR_BAD_ARG
    assert b"positive" in _abi.lib().msosm_last_error()


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU path")
def test_no_device_is_reported_not_crashed():
    assert _abi.lib().msosm_device_count() == 0
    bw = np.array([16e6], np.float32)
    dm = np.array([5.0], np.float32)
    f0 = np.array([1242e6], np.float32)
    h = ctypes.c_void_p()
    st = _abi.lib().msosm_dedisp_create(bw.ctypes.data, dm.ctypes.data, f0.ctypes.data, 1, 1024, 4, 0, 0,
                                        ctypes.byref(h))
    assert st == _abi.ERR_NO_DEVICE and not h.value


def test_tensor_path_rejects_other_fft_sizes():
    # checked before any device work, so this holds with or without a GPU
    bw = np.array([16e6], np.float32)
    dm = np.array([5.0], np.float32)
    f0 = np.array([1242e6], np.float32)
    h = ctypes.c_void_p()
    st = _abi.lib().msosm_dedisp_create(bw.ctypes.data, dm.ctypes.data, f0.ctypes.data, 1, 2048, 4, 0,
                                        _abi.FLAG_TENSOR_F16, ctypes.byref(h))
    assert st == _abi.ERR_UNSUPPORTED and not h.value
    assert b"4096" in _abi.lib().msosm_last_error()
    st = _abi.lib().msosm_dedisp_create(bw.ctypes.data, dm.ctypes.data, f0.ctypes.data, 1, 4096, 4, 0,
                                        _abi.FLAG_TENSOR_F16 | _abi.FLAG_TENSOR_BF16, ctypes.byref(h))
    assert st == _abi.ERR_BAD_ARG and not h.value


@pytest.mark.parametrize("log2n", [12, 13])
def test_tensor_layout_tables(log2n):
    # host mirror of tc_pos (tc_layout.hpp) is a permutation of the bins, and
    # the gather's thread mapping (W warps) puts the bin pairs of one warp
    # store in one 128-byte core matrix of the MN-major operand
    N = 1 << log2n
    W = (N // 64) // 8

    def tc_pos(b):
        k1, k2 = b & 63, b >> 6
        u = (k1 >> 3) * W + (k2 >> 3)
        l = (k2 & 7) * 4 + ((k1 & 7) >> 1)
        return u * 64 + l * 2 + (k1 & 1)

    def mn_off(r, k):
        return (r >> 3) * 128 + (k >> 3) * 2048 + (k & 7) * 16 + (r & 7) * 2

    pos = np.array([tc_pos(b) for b in range(N)])
    assert np.array_equal(np.sort(pos), np.arange(N))
    inv = np.argsort(pos)
    for j in range(8):
        for w in range(W):
            offs = []
            for lane in range(32):
                b = inv[(j * W + w) * 64 + 2 * lane]
                k1, k2 = b & 63, b >> 6
                offs.append(mn_off(k1, k2))
                assert inv[(j * W + w) * 64 + 2 * lane + 1] == b + 1
            offs = np.array(offs)
            assert np.array_equal(np.sort(offs), offs.min() + 4 * np.arange(32))
            assert offs.min() % 128 == 0
    # every operand element (128 rows, K = 2 N / 64) lies inside its buffer
    K = 2 * (N // 64)
    assert max(mn_off(r, k) for r in range(128) for k in range(K)) < 128 * K * 2


@pytest.mark.parametrize("k", range(len(META["msosm"])))
def test_prepare_matches_reference(k):
    s = META["msosm"][k]
    Nd = prepare.nd(s["bw"], s["dm"], s["f0"])
    assert Nd == s["Nd"]
    assert prepare.msosm_min_order(Nd) == s["M_min"]
    dc, dp = prepare.segmentation(s["bw"], s["dm"], s["f0"], s["M"])
    assert dc == s["delaycount"]
    np.testing.assert_array_equal(dp, ARR[f"msosm{k}_delay_points"].astype(np.int32))


def test_concurrent_grid_segmentation_matches_reference():
    s = META["concurrent"]
    M = s["M_common"]
    dps = ARR["concurrent_delay_points"].astype(np.int32).reshape(len(s["dm"]), 2 * M)
    for i, dm in enumerate(s["dm"]):
        assert prepare.nd(s["bw"], dm, s["f0"]) == s["Nd"][i]
        dc, dp = prepare.segmentation(s["bw"], dm, s["f0"], M)
        assert dc == s["delaycount"][i]
        np.testing.assert_array_equal(dp, dps[i])


@pytest.mark.parametrize("k", range(len(META["osm"])))
def test_osm_order_matches_reference(k):
    s = META["osm"][k]
    assert prepare.nd(s["bw"], s["dm"], s["f0"]) == s["Nd"]
    assert prepare.osm_min_order(s["Nd"]) == s["M_min"]


def test_prepare_matches_oracle_on_a_dm_grid():
    # the 256-trial grid over DM 0-100 at 16 MHz / 1242 MHz with FFT 4096,
    # plus a 64 MHz band: integers must agree everywhere
    for bw, f0, M, dms in [(16e6, 1242e6, 2048, np.linspace(0, 100, 256)),
                           (64e6, 1368e6, 4096, np.linspace(0, 200, 97))]:
        for dm in dms.astype(np.float32):
            assert prepare.nd(bw, dm, f0) == O.nd(bw, dm, f0)
            dc, dp = prepare.segmentation(bw, dm, f0, M)
            odc, odp = O.segmentation(bw, dm, f0, M)
            assert dc == odc
            np.testing.assert_array_equal(dp, odp)


def test_dm_zero_has_no_delays():
    dc, dp = prepare.segmentation(16e6, 0.0, 1242e6, 2048)
    assert dc == 0 and not dp.any()


def _fold_from_planner(period, fs, size, chunks, Nd, I):
    pl = prepare.FoldPlanner(period, fs, Nd)
    per = {}
    for c in range(chunks):
        dest, _ = pl.chunk(size)
        for i in np.nonzero(dest >= 0)[0]:
            d = int(dest[i])
            per.setdefault(d >> 32, {})[d & 0xFFFFFFFF] = I[c * size + i]
    ps = int(np.float32(period) * np.float32(fs))
    raw = np.zeros(ps)
    for p, m in per.items():
        if len(m) == ps:
            for ph, v in m.items():
                raw[ph] += v
    return raw


@pytest.mark.parametrize("case", [
    (0.01234, 1e4, 1000, 20, 300),
    (0.01234, 1e4, 97, 60, 300),
    (0.00531, 2e4, 512, 40, 1000),
    (0.0031, 16e4, 2048, 30, 900),
    (0.00123, 1e5, 123, 50, 100),   # chunks shorter than a period
    (0.0005, 1e5, 1000, 20, 10),    # several periods per chunk
])
def test_fold_planner_equals_fold_gpu_state_machine(case):
    period, fs, size, chunks, Nd = case
    rng = np.random.default_rng(7)
    I = rng.random(size * chunks)
    raw = _fold_from_planner(period, fs, size, chunks, Nd, I)
    f = O.Fold(period, fs, size, -1, accumulate_float=False)
    f.discard_samples(Nd)
    for c in range(chunks):
        f.fold_data(I[c * size:(c + 1) * size])
    np.testing.assert_allclose(raw, f.fold_data_bins(), rtol=1e-12, atol=1e-12)


def test_fold_planner_deferred_skip_at_chunk_end():
    # period 10.5 samples: a skip every other period; chunks of 21 end
    # exactly where a skip is due, which the reference defers
    raw = _fold_from_planner(0.00105, 1e4, 21, 40, 30, np.arange(21 * 40, dtype=float))
    f = O.Fold(0.00105, 1e4, 21, -1, accumulate_float=False)
    f.discard_samples(30)
    I = np.arange(21 * 40, dtype=float)
    for c in range(40):
        f.fold_data(I[c * 21:(c + 1) * 21])
    np.testing.assert_allclose(raw, f.fold_data_bins())
