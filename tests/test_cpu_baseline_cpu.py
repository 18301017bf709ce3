"""The timed CPU baseline (oracle/cpu_fp32.py: the reference's MS-OSM and OSM
in FP32 on the host cores) computes what the FP64 oracle computes, to FP32
rounding: series within 1e-6 relative RMS per trial, and its Fold_GPU
profiles within 1e-5."""
import numpy as np

import oracle as O
import cpu_fp32 as C

BW, F0 = 16e6, 1242e6


def rel(a, b):
    return np.sqrt(np.sum(np.abs(a - b) ** 2, axis=-1) / np.sum(np.abs(b) ** 2, axis=-1))


def test_fp32_msosm_matches_fp64_oracle():
    dms = np.linspace(0.0, 60.0, 6).astype(np.float32)
    rng = np.random.default_rng(0)
    c = C.MsosmFP32(BW, dms, F0, 2048, 8, period=0.00031, time_bin=32, threads=4)
    o = O.Dedisp(BW, dms, F0, 2048, 8)
    folds = [O.Fold(0.00031, BW, 8 * c.M, 32) for _ in dms]
    for f in folds:
        f.discard_samples(max(o.Nd))
    for _ in range(10):
        x = ((rng.standard_normal(8 * c.M) + 1j * rng.standard_normal(8 * c.M)) * 100).astype(np.complex64)
        y = c.filter(x, keep_series=True)
        r = o.filter(x.astype(np.complex128))
        assert rel(y, r).max() < 1e-6
        for f, row in zip(folds, r):
            f.fold_data(np.abs(row) ** 2)
    p, pr = c.profiles(), np.stack([f.fold_data_bins() for f in folds])
    assert np.abs(pr).max() > 0
    assert rel(p, pr).max() < 1e-5
    c.close()


def test_fp32_osm_matches_fp64_oracle():
    rng = np.random.default_rng(1)
    c = C.MsosmFP32(BW, [0.5, 3.0], F0, 0, 4, osm=True, threads=2)
    o = O.Dedisp(BW, [0.5, 3.0], F0, 0, 4, osm=True)
    assert c.M == o.M
    for _ in range(3):
        x = ((rng.standard_normal(4 * c.M) + 1j * rng.standard_normal(4 * c.M)) * 100).astype(np.complex64)
        assert rel(c.filter(x, keep_series=True), o.filter(x.astype(np.complex128))).max() < 1e-6
    c.close()
