"""The FP64 oracle pinned against the reference's own host code.

Fixtures in tests/golden/ were produced by the reference's filter design,
segmentation, Fold_GPU and simulator compiled from its sources
(tests/golden/make_golden.py).  Integer results must match exactly; float
results to the rounding of the reference's single-precision storage.
"""
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
META = json.load(open(os.path.join(HERE, "golden", "reference_host.json")))
ARR = np.load(os.path.join(HERE, "golden", "reference_host.npz"))


def _c(a):
    return a.astype(np.float64).view(np.complex128)


@pytest.mark.parametrize("k", range(len(META["msosm"])))
def test_msosm_prepare_matches_reference(k):
    s = META["msosm"][k]
    Nd = O.nd(s["bw"], s["dm"], s["f0"])
    assert Nd == s["Nd"]
    assert O.msosm_min_order(Nd) == s["M_min"]
    M = s["M_min"] if s["fftpoint"] == 0 else max(s["fftpoint"] // 2, s["M_min"])
    assert M == s["M"]
    dc, dp = O.segmentation(s["bw"], s["dm"], s["f0"], M)
    assert dc == s["delaycount"]
    np.testing.assert_array_equal(dp, ARR[f"msosm{k}_delay_points"].astype(np.int32))
    H = O.dedisp_params(s["bw"], s["dm"], s["f0"], M)
    Hr = _c(ARR[f"msosm{k}_H"])
    rel = np.sqrt(np.mean(np.abs(H - Hr) ** 2) / np.mean(np.abs(H) ** 2))
    assert rel < 1e-6, rel


def test_concurrent_prepare_matches_reference():
    s = META["concurrent"]
    d = O.Dedisp(s["bw"], s["dm"], s["f0"], s["fftpoint"], count=4)
    assert d.M == s["M_common"]
    assert d.Nd == s["Nd"]
    assert d.delaycount == s["delaycount"]
    M = d.M
    dps = ARR["concurrent_delay_points"].astype(np.int32).reshape(len(s["dm"]), 2 * M)
    Hs = _c(ARR["concurrent_H"]).reshape(len(s["dm"]), 2 * M)
    for i, dm in enumerate(s["dm"]):
        dc, dp = O.segmentation(s["bw"], dm, s["f0"], M)
        np.testing.assert_array_equal(dp, dps[i])
        H = O.dedisp_params(s["bw"], dm, s["f0"], M)
        rel = np.sqrt(np.mean(np.abs(H - Hs[i]) ** 2) / np.mean(np.abs(H) ** 2))
        assert rel < 1e-6


@pytest.mark.parametrize("k", range(len(META["osm"])))
def test_osm_prepare_matches_reference(k):
    s = META["osm"][k]
    Nd = O.nd(s["bw"], s["dm"], s["f0"])
    assert Nd == s["Nd"]
    assert O.osm_min_order(Nd) == s["M_min"]
    M = s["M_min"] if s["fftpoint"] == 0 else max(s["fftpoint"] // 2, s["M_min"])
    assert M == s["M"]
    H = O.dedisp_params(s["bw"], s["dm"], s["f0"], M)
    Hr = _c(ARR[f"osm{k}_H"])
    rel = np.sqrt(np.mean(np.abs(H - Hr) ** 2) / np.mean(np.abs(H) ** 2))
    assert rel < 1e-6


@pytest.mark.parametrize("k", range(len(META["fold"])))
def test_fold_matches_reference_bit_exact(k):
    s = META["fold"][k]
    I = ARR[f"fold{k}_intensity"].astype(np.float64)
    f = O.Fold(s["period"], s["fs"], s["size"], s["time_bin"], accumulate_float=True)
    assert f.period_samples == s["period_samples"]
    assert f.time_bin == s["time_bin_out"]
    f.discard_samples(s["Nd"])
    for c in range(s["chunks"]):
        f.fold_data(I[c * s["size"]:(c + 1) * s["size"]])
    np.testing.assert_array_equal(f.fold_data_bins().astype(np.float32), ARR[f"fold{k}_folded"])
    g = O.Fold(s["period"], s["fs"], s["size"], s["time_bin"], accumulate_float=False)
    g.discard_samples(s["Nd"])
    for c in range(s["chunks"]):
        g.fold_data(I[c * s["size"]:(c + 1) * s["size"]])
    np.testing.assert_allclose(g.fold_data_bins(), ARR[f"fold{k}_folded"], rtol=1e-5)


def test_simulator_matches_reference():
    s = META["simulate"]
    x = O.simulate_two_spike(s["bw"], s["dm"], s["f0"], s["period"], s["repeat"])
    xr = _c(ARR["simulate_signal"])
    assert x.size == s["Np"] * s["repeat"]
    assert np.abs(x - xr).max() / np.abs(xr).max() < 1e-6
