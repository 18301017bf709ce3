"""PSRDADA reader on the host (no GPU): header fields, readCount and the
frame de-interleave against the reference's own PSRDADA class (golden
fixture from tests/golden/make_dada_golden.py), the writer/reader round trip,
and the error cases the reference leaves undefined."""
import hashlib
import json
import os

import numpy as np
import pytest

from msosm_gpu_b200 import MsosmError, _abi, psrdada as P

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = json.load(open(os.path.join(HERE, "golden", "reference_dada.json")))


def file_bytes(case) -> bytes:
    # the same construction as tests/golden/make_dada_golden.py
    rng = np.random.default_rng(case["seed"])
    hdr = case["header"].encode()
    body = rng.integers(0, 65536, size=2 * case["pairs"], dtype=np.uint16).tobytes()
    tail = rng.integers(0, 256, size=case["trailing"], dtype=np.uint8).tobytes()
    return hdr + b"\0" * (4096 - len(hdr)) + body + tail


@pytest.mark.parametrize("k", range(len(CASES)))
def test_reader_matches_reference_psrdada(k, tmp_path):
    c = CASES[k]
    e = c["expected"]
    path = str(tmp_path / "x.dada")
    open(path, "wb").write(file_bytes(c))
    f = P.PSRDADA(path)
    assert (f.bw, f.fc) == (e["bw"], e["fc"])
    for key in ("nbit", "nchan", "ndim", "npol"):
        if e[key] is None:
            assert getattr(f, key) == 0  # absent key: 0 here, uninitialised in the reference
        else:
            assert getattr(f, key) == e[key], key
    assert f.filesize == e["filesize"]
    f.initBuffer(c["n"])
    assert (f.readCount, f.frameCount) == (e["readCount"], e["frameCount"])
    p1, p2 = [], []
    for _ in range(c["reads"]):
        f.readSamples()
        p1.append(f.pol1_in.copy())
        p2.append(f.pol2_in.copy())
    assert hashlib.sha256(np.concatenate(p1).tobytes()).hexdigest() == e["pol1_sha256"]
    assert hashlib.sha256(np.concatenate(p2).tobytes()).hexdigest() == e["pol2_sha256"]
    f.close()


def test_write_read_round_trip_and_end_of_file(tmp_path):
    rng = np.random.default_rng(7)
    n = 3 * 2048
    a = rng.integers(0, 65536, (n, 2), dtype=np.uint16)
    b = rng.integers(0, 65536, (n, 2), dtype=np.uint16)
    path = str(tmp_path / "obs.dada")
    P.write_dada(path, a, b, bw_mhz=32, freq_mhz=1400)
    f = P.PSRDADA(path)
    assert (f.bw, f.fc, f.npol) == (32.0, 1400.0, 2)
    assert f.outfileName == str(tmp_path / "obs_dedisp_folded.txt")
    f.initBuffer(2048)
    assert f.readCount == 3
    for r in range(3):
        f.readSamples()
        assert np.array_equal(f.pol1_in, a[r * 2048:(r + 1) * 2048])
        assert np.array_equal(f.pol2_in, b[r * 2048:(r + 1) * 2048])
    with pytest.raises(MsosmError) as ei:
        f.readSamples()  # the reference reads past the end silently
    assert ei.value.status == _abi.ERR_STATE
    with pytest.raises(ValueError):
        f.initBuffer(1000)


def test_open_errors(tmp_path):
    with pytest.raises(MsosmError):
        P.PSRDADA(str(tmp_path / "missing.dada"))
    short = tmp_path / "short.dada"
    short.write_bytes(b"BW 16\n")
    with pytest.raises(MsosmError):
        P.PSRDADA(str(short))
