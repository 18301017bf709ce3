"""Many observations in one launch (msosm_batch / DedispBatch): observations
of different length, band, trial grid and FFT size (4096, 8192, 16384)
dedispersed by one persistent tensor-core launch per kernel group, every observation's series
and folded profiles against the FP64 oracle (the tensor path's bounds) and
against the same observation run through its own handle (the batch keeps
each handle's own work items, so the two agree to rounding).  An FP32 handle in
the same batch runs its own launch inside the batch call."""
import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import DedispBatch, Dedisperser

pytestmark = pytest.mark.gpu

SERIES_TOL, FOLD_TOL = 1.5e-3, 1e-4

OBS = [  # bw, f0, dms, fftpoint, count, precision, period (smears short enough to fold whole periods)
    (16e6, 1242e6, [0.0, 3.0, 8.0], 4096, 12, "fp16", 0.00031),
    (64e6, 1368e6, [0.5, 2.0], 8192, 7, "fp16", 0.0002),
    (32e6, 1384e6, [1.0, 4.0, 6.0, 8.0], 4096, 12, "fp16", 0.00045),
    (16e6, 1242e6, [2.0, 9.0], 4096, 9, "fp16", 0.00029),
    (4e6, 1098e6, [3.0, 30.0], 2048, 6, "fp32", 0.0013),
    (16e6, 1242e6, [1.0, 5.0], 16384, 3, "fp16", 0.0011),
]


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def make(o, nbins=64):
    bw, f0, dms, fp, count, prec, period = o
    d = Dedisperser(bw, dms, f0, fp, count, precision=prec)
    d.fold_init(period, bw, time_bin=nbins, discard_Nd=int(d.Nd.max()), detect="power")
    return d


def test_batch_matches_oracle_and_own_handles():
    rng = np.random.default_rng(5)
    calls = 4
    batch_h = [make(o) for o in OBS]
    solo_h = [make(o) for o in OBS]
    b = DedispBatch(batch_h)
    info = b.info()
    assert info["groups"] == 3 and info["launches_per_call"] == 4
    orc = [O.Dedisp(o[0], o[2], o[1], o[3], o[4]) for o in OBS]
    folds = [[O.Fold(o[6], o[0], d.block_samples, 64) for _ in o[2]] for o, d in zip(OBS, batch_h)]
    for fl, d in zip(folds, batch_h):
        for f in fl:
            f.discard_samples(int(d.Nd.max()))
    worst = {}
    for c in range(calls):
        xs = [((rng.standard_normal(d.block_samples) + 1j * rng.standard_normal(d.block_samples)) * 300)
              .astype(np.complex64) for d in batch_h]
        b.filter_block(xs)
        for i, (d, s, o, x) in enumerate(zip(batch_h, solo_h, orc, xs)):
            s.filter_block(x)
            ref = o.filter(x.astype(np.complex128))
            y, ys = d.get_output(), s.get_output()
            for t in range(d.numDMs):
                folds[i][t].fold_data(np.abs(ref[t]) ** 2)
                tol = SERIES_TOL if OBS[i][5] != "fp32" else 2e-5
                e = rel_rms(y[t], ref[t])
                assert e < tol, (i, t, c, e)
                # the same work items as the handle's own calls: equal to rounding
                assert rel_rms(y[t], ys[t]) < 1e-6, (i, t, c, rel_rms(y[t], ys[t]))
                worst[i] = max(worst.get(i, 0.0), e)
    for i, (d, s) in enumerate(zip(batch_h, solo_h)):
        p, ps = d.get_profiles().astype(np.float64), s.get_profiles().astype(np.float64)
        pr = np.stack([f.fold_data_bins() for f in folds[i]])
        assert d.folded_periods() == s.folded_periods() > 0
        for t in range(d.numDMs):
            assert rel_rms(p[t], pr[t]) < (FOLD_TOL if OBS[i][5] != "fp32" else 2e-5), (i, t)
            assert rel_rms(p[t], ps[t]) < 1e-6, (i, t)
    b.synchronize()
    b.close()
    # the handles go back to their own streams and keep working
    x = np.zeros(batch_h[0].block_samples, np.complex64)
    batch_h[0].filter_block(x)
    batch_h[0].synchronize()


def test_batch_rejects_a_handle_twice():
    from msosm_gpu_b200 import _abi
    d = make(OBS[0])
    with pytest.raises(_abi.MsosmError):
        DedispBatch([d, d])


def test_batch_groups_by_precision_and_size():
    # bf16 members at FFT 8192 and 16384 and an f16 member at 16384 form three
    # kernel groups; each member's profiles equal its own handle's to
    # rounding, and its series is within the bf16 / f16 bound of the oracle
    obs = [(16e6, 1242e6, [1.0, 6.0], 8192, 6, "bf16", 0.0011),
           (16e6, 1242e6, [2.0, 5.0], 16384, 3, "bf16", 0.0011),
           (16e6, 1242e6, [0.5, 4.0], 16384, 3, "fp16", 0.0011)]
    batch_h = [make(o) for o in obs]
    solo_h = [make(o) for o in obs]
    b = DedispBatch(batch_h)
    assert b.info()["groups"] == 3
    orc = [O.Dedisp(o[0], o[2], o[1], o[3], o[4]) for o in obs]
    rng = np.random.default_rng(9)
    for c in range(4):
        xs = [((rng.standard_normal(d.block_samples) + 1j * rng.standard_normal(d.block_samples)) * 300)
              .astype(np.complex64) for d in batch_h]
        b.filter_block(xs)
        for d, s, o, x, ob in zip(batch_h, solo_h, orc, xs, obs):
            s.filter_block(x)
            ref = o.filter(x.astype(np.complex128))
            y, ys = d.get_output(), s.get_output()
            for t in range(d.numDMs):
                assert rel_rms(y[t], ys[t]) < 1e-6
                assert rel_rms(y[t], ref[t]) < (1e-2 if ob[5] == "bf16" else SERIES_TOL)
    for d, s in zip(batch_h, solo_h):
        assert d.folded_periods() == s.folded_periods() > 0
        p, ps = d.get_profiles().astype(np.float64), s.get_profiles().astype(np.float64)
        for t in range(d.numDMs):
            assert rel_rms(p[t], ps[t]) < 1e-6
    b.close()
