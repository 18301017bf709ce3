"""FFT sizes above one thread block (four-step path): OSM at 2^18 points (the
single-DM DM-50 configuration's overlap-save run, 16 MHz at 1250 MHz) and
MS-OSM at 2^15..2^20 against the FP64 oracle, the reference's own
OSM_GPU_BATCH, and the filter design against the oracle."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import Dedisperser

pytestmark = pytest.mark.gpu

BW, F0 = 16e6, 1242e6
RTOL = 2e-5


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def u16(n, seed):
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.standard_normal((n, 2)) * 1000) + 32768, 1, 65535).astype(np.uint16)


def pair(dms, fftpoint, count, calls, osm=False, seed=0):
    d = Dedisperser(BW, dms, F0, fftpoint, count, osm=osm)
    o = O.Dedisp(BW, dms, F0, fftpoint, count, osm=osm)
    assert (d.M, d.count) == (o.M, o.count)
    x = u16(d.block_samples * calls, seed)
    ours, ref = [], []
    for c in range(calls):
        blk = x[c * d.block_samples:(c + 1) * d.block_samples]
        d.filter_block(blk)
        ours.append(d.get_output())
        ref.append(o.filter(O.decode_uint16(blk)))
    return np.concatenate(ours, 1), np.concatenate(ref, 1), d, x


@pytest.mark.parametrize("fftpoint,dms,osm", [
    (32768, [5.0], True),
    (0, [50.0], True),              # OSM minimum for DM 50: 2^18 points
    (32768, [100.0, 300.0], False),
    (1 << 20, [50.0], False),
])
def test_large_fft_matches_oracle(fftpoint, dms, osm):
    ours, ref, d, _ = pair(dms, fftpoint, 1 if fftpoint >= (1 << 18) or fftpoint == 0 else 2, 3, osm)
    assert d.fftpoint > 16384
    for i in range(len(dms)):
        assert rel_rms(ours[i], ref[i]) < RTOL, (i, rel_rms(ours[i], ref[i]))


def test_large_filter_design_matches_oracle():
    d = Dedisperser(BW, [50.0], F0, 0, 1, osm=True)
    assert d.fftpoint == 1 << 18
    H = d.dedisp_params(0)
    Ho = O.dedisp_params(BW, 50.0, F0, d.M)
    assert rel_rms(H, Ho) < RTOL


def test_osm_2p18_matches_reference_osm_gpu_batch():
    if not os.path.exists(O.REF_GPU_RUNNER):
        pytest.skip("reference runner not built")
    calls, dm = 3, 50.0
    ours, _, d, x = pair([dm], 0, 1, calls, osm=True, seed=5)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.u16"), os.path.join(td, "out.bin")
        x.tofile(fin)
        r = subprocess.run([O.REF_GPU_RUNNER, "osm", "0", "1", str(calls), str(BW), str(dm), str(F0), fin, fout],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        rec = O.read_records(fout)
    assert int(rec["M"][0]) == d.M
    ref = rec["out"].astype(np.float64).view(np.complex128)
    assert rel_rms(ours[0], ref) < 1e-4, rel_rms(ours[0], ref)


def test_large_fft_fold_matches_oracle():
    dms, fftpoint, count, calls, period, tb = [100.0, 300.0], 32768, 2, 6, 0.0011, 64
    d = Dedisperser(BW, dms, F0, fftpoint, count, series=False)
    nd = 20000  # two periods discarded (the DM-300 smear would discard the whole stream)
    d.fold_init(period, BW, time_bin=tb, discard_Nd=nd, detect="amplitude")
    o = O.Dedisp(BW, dms, F0, fftpoint, count)
    x = u16(d.block_samples * calls, 9)
    ser = []
    for c in range(calls):
        blk = x[c * d.block_samples:(c + 1) * d.block_samples]
        d.filter_block(blk)
        ser.append(o.filter(O.decode_uint16(blk)))
    ser = np.concatenate(ser, 1)
    prof = d.get_profiles()
    assert d.folded_periods() > 0
    for i in range(len(dms)):
        f = O.Fold(period, BW, d.block_samples, tb)
        f.discard_samples(nd)
        for c in range(calls):
            f.fold_data(np.abs(ser[i, c * d.block_samples:(c + 1) * d.block_samples]))
        assert rel_rms(prof[i], f.fold_data_bins()) < RTOL
