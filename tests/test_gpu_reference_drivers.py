"""The reference's own driver programs, unmodified, built against the drop-in
headers and libmsosm_b200.so (oracle/Makefile `drivers`, into
oracle/_ref/drivers/), run on the GPU.

check_msosm.cpp (the reference's MS-OSM check): one DM (128 MHz at 1 GHz,
DM 75) over its two-spike simulated signal in calls of 4 blocks, uint16
output, and a plot of |x| of the last period.  The headless plot helper of
include/compat/globals.h writes that plotted series to MSOSM_PLOT_DUMP; it
must equal what the Python binding computes from the same signal through the
same library (bit for bit: same inputs, same kernels).
test_processing_speed_msosm.cpp must run to completion."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200 import Dedisperser
from msosm_gpu_b200.simulator import SimulatedComplexSignal

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRV = os.path.join(ROOT, "oracle", "_ref", "drivers")


def read_dump(path):
    out = []
    with open(path, "rb") as f:
        while True:
            head = f.read(40)
            if len(head) < 40:
                break
            name = head[:32].rstrip(b"\0").decode()
            n = int(np.frombuffer(head[32:40], np.uint64)[0])
            out.append((name, np.frombuffer(f.read(4 * n), np.float32)))
    return out


@pytest.mark.skipif(not os.path.exists(os.path.join(DRV, "check_msosm")), reason="drivers not built")
def test_check_msosm_runs_unchanged_and_matches_python_binding():
    # calls of 4 blocks, so that the plotted last period is almost all output
    # (the driver's buffer holds signal_size + calls elements; calls of 32
    # blocks would leave most of that period unwritten)
    bw, dm, f0, period, count = 128e6, 75.0, 1e9, 0.002048, 4
    compare = 1 << 24
    with tempfile.TemporaryDirectory() as td:
        dump = os.path.join(td, "plot.bin")
        env = dict(os.environ, MSOSM_PLOT_DUMP=dump)
        r = subprocess.run([os.path.join(DRV, "check_msosm"), "--compare", str(compare), "--batch", str(count)],
                           capture_output=True,
                           text=True, timeout=600, env=env, cwd=td)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        recs = read_dump(dump)
    assert [n for n, _ in recs] == ["plot_abs_u16"]
    plotted = recs[0][1]
    # the driver's own arithmetic: block_size = period * bw samples per period,
    # inputSize periods of signal, calls of count * M samples each written to
    # output + k * (process_len + 1), then |x| of block_size values from
    # output + (inputSize - 1) * block_size
    sig = SimulatedComplexSignal(bw, dm, f0, period, "uint16")
    block = int(np.float32(period) * np.float32(bw))
    input_size = compare // block
    sig.generate_pulsar_signal(input_size, False, 0.0, False)
    d = Dedisperser(bw, [dm], f0, 0, count)
    plen = d.block_samples
    calls = sig.signal_size // plen
    out = np.zeros((sig.signal_size + calls, 2), np.uint16)
    for k in range(calls):
        d.filter_block(sig.signal_u16[k * plen:(k + 1) * plen])
        d.get_output(out=out[k * (plen + 1):(k + 1) * (plen + 1)], dtype=np.uint16)
    seg = out[(input_size - 1) * block:(input_size - 1) * block + block].astype(np.int64)
    dec = np.where(seg == 0, 0, seg - 32768).astype(np.float32)
    mine = np.hypot(dec[:, 0], dec[:, 1]).astype(np.float32)
    assert plotted.size == block
    np.testing.assert_array_equal(plotted, mine)
    assert np.count_nonzero(mine) > block // 2


@pytest.mark.skipif(not os.path.exists(os.path.join(DRV, "test_processing_speed_msosm")),
                    reason="drivers not built")
def test_reference_speed_test_runs_unchanged():
    r = subprocess.run([os.path.join(DRV, "test_processing_speed_msosm"), "--compare", str(1 << 22),
                        "--batch", "16", "--repeat", "3"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Time taken (ms)" in r.stdout
