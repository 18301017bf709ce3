"""PSRDADA baseband files and the two-polarisation fold pipeline.

``PSRDADA`` mirrors the reference's reader (psrdada/include/psrdada.h:17-43):
the 4096-byte header's BW / FREQ / NBIT / NCHAN / NDIM / NPOL, ``initBuffer``
and ``readSamples`` de-interleaving the 2048-sample frames of the two
polarisations; the file access itself is the C ABI's ``msosm_dada_*``.
``fold_file`` is the reference's ``msosm_psrdada`` driver
(msosm_psrdada.cpp:92-144): one MS-OSM dedisperser per polarisation,
sqrt(|a|^2 + |b|^2) on the device, Fold_GPU folding, the leading reads whose
first sample is blank skipped.  ``write_dada`` writes files of the same
format (for tests and simulations).

    python -m msosm_gpu_b200.psrdada --file obs.dada --dm 750 --period 0.032768
"""
from __future__ import annotations

import argparse
import ctypes
import os
import queue
import threading
import time
from typing import Optional

import numpy as np

from . import _abi
from ._abi import check, lib

HEADER_BYTES = 4096
FRAME_SAMPLES = 2048


class DadaInfo(ctypes.Structure):
    _fields_ = [
        ("bw", ctypes.c_float),
        ("fc", ctypes.c_float),
        ("nbit", ctypes.c_int),
        ("nchan", ctypes.c_int),
        ("ndim", ctypes.c_int),
        ("npol", ctypes.c_int),
        ("have", ctypes.c_uint),
        ("filesize", ctypes.c_ulonglong),
    ]


class PSRDADA:
    """A PSRDADA file: header fields, then reads of n samples per polarisation."""

    def __init__(self, filename: str):
        self.infileName = filename
        h = ctypes.c_void_p()
        check(lib().msosm_dada_open(filename.encode(), ctypes.byref(h)))
        self._h = h
        info = DadaInfo()
        check(lib().msosm_dada_get_info(self._h, ctypes.byref(info)))
        hdr = ctypes.create_string_buffer(HEADER_BYTES)
        check(lib().msosm_dada_get_header(self._h, hdr))
        self.headerBuffer = hdr.raw
        self.bw, self.fc = float(np.float32(info.bw)), float(np.float32(info.fc))
        self.nbit, self.nchan, self.ndim, self.npol = info.nbit, info.nchan, info.ndim, info.npol
        self.filesize = int(info.filesize)
        self.have_bw = bool(info.have & 1)
        self.have_freq = bool(info.have & 2)
        self.outfileName = os.path.splitext(filename)[0] + "_dedisp_folded.txt"
        self.pol1_in = self.pol2_in = None
        self.frameCount = 0
        self.readCount = 0

    def initBuffer(self, n: int) -> None:
        if n <= 0 or n % FRAME_SAMPLES:
            raise ValueError(f"n must be a multiple of frameSamples ({FRAME_SAMPLES})")
        self.pol1_in = np.zeros((n, 2), np.uint16)
        self.pol2_in = np.zeros((n, 2), np.uint16)
        self.frameCount = n // FRAME_SAMPLES
        c = ctypes.c_ulong()
        check(lib().msosm_dada_read_count(self._h, n, ctypes.byref(c)))
        self.readCount = int(c.value)

    def readSamples(self) -> None:
        n = self.pol1_in.shape[0]
        check(lib().msosm_dada_read(self._h, n, self.pol1_in.ctypes.data, self.pol2_in.ctypes.data))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().msosm_dada_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_dada(path: str, pol1: np.ndarray, pol2: np.ndarray, bw_mhz: float = 16.0, freq_mhz: float = 1250.0,
               extra: Optional[dict] = None) -> None:
    """Write uint16 offset-binary pairs (arrays of shape (n, 2), n a multiple of
    2048) of two polarisations as a PSRDADA file with a 4096-byte header."""
    pol1 = np.ascontiguousarray(pol1, np.uint16).reshape(-1, 2)
    pol2 = np.ascontiguousarray(pol2, np.uint16).reshape(-1, 2)
    n = pol1.shape[0]
    if pol2.shape[0] != n or n % FRAME_SAMPLES:
        raise ValueError("both polarisations need the same length, a multiple of 2048")
    keys = {"HDR_VERSION": "1.0", "HDR_SIZE": str(HEADER_BYTES), "BW": f"{bw_mhz:g}", "FREQ": f"{freq_mhz:g}",
            "NBIT": "16", "NCHAN": "1", "NDIM": "2", "NPOL": "2"}
    if extra:
        keys.update({k: str(v) for k, v in extra.items()})
    text = "".join(f"{k:<15} {v}\n" for k, v in keys.items()).encode()
    if len(text) >= HEADER_BYTES:
        raise ValueError("header longer than 4096 bytes")
    frames = np.stack([pol1.reshape(-1, FRAME_SAMPLES, 2), pol2.reshape(-1, FRAME_SAMPLES, 2)], 1)
    with open(path, "wb") as f:
        f.write(text + b"\0" * (HEADER_BYTES - len(text)))
        f.write(frames.tobytes())


class _PinnedPairs:
    """``n`` pairs of pinned host buffers of `samples` uint16 pairs."""

    def __init__(self, n: int, samples: int):
        self._ptrs = []
        self.pairs = []
        for _ in range(n):
            pair = []
            for _ in range(2):
                p = ctypes.c_void_p()
                check(lib().msosm_host_alloc(samples * 4, 1, ctypes.byref(p)))
                self._ptrs.append(p)
                buf = (ctypes.c_uint16 * (2 * samples)).from_address(p.value)
                pair.append(np.ctypeslib.as_array(buf).reshape(samples, 2))
            self.pairs.append(tuple(pair))

    def close(self) -> None:
        for p in self._ptrs:
            lib().msosm_host_free(p, 1)
        self._ptrs, self.pairs = [], []


def _reads(f: PSRDADA, overlap: bool, depth: int = 3):
    """Yields (pol1, pol2) of every whole read of the file in order.  With
    ``overlap`` a reader thread fills `depth` pinned buffer pairs ahead of
    the consumer (file I/O under the device work; a pair is handed back when
    the consumer asks for the next one, after its filter calls have copied it
    to the device)."""
    n = f.pol1_in.shape[0]
    if not overlap:
        for _ in range(f.readCount):
            f.readSamples()
            yield f.pol1_in, f.pol2_in
        return
    bufs = _PinnedPairs(depth, n)
    free: "queue.Queue" = queue.Queue()
    ready: "queue.Queue" = queue.Queue()
    for b in bufs.pairs:
        free.put(b)
    stop = threading.Event()

    def reader():
        try:
            for _ in range(f.readCount):
                b = free.get()
                if stop.is_set():
                    break
                check(lib().msosm_dada_read(f._h, n, b[0].ctypes.data, b[1].ctypes.data))
                ready.put(b)
            ready.put(None)
        except BaseException as e:  # handed to the consumer
            ready.put(e)

    t = threading.Thread(target=reader, daemon=True)
    t.start()
    try:
        while True:
            b = ready.get()
            if b is None:
                break
            if isinstance(b, BaseException):
                raise b
            yield b
            free.put(b)
    finally:
        stop.set()
        free.put(None)
        t.join()
        bufs.close()


def fold_file(filename: str, dm: float, period: float, fftpoint: int = 2097152, count: int = 1,
              time_bin: int = 1024, precision: str = "fp32", write: bool = True, overlap: bool = True,
              stats: Optional[dict] = None) -> np.ndarray:
    """The two-polarisation pipeline of msosm_psrdada.cpp:92-144 on a
    PSRDADA file; returns the folded profile (time_bin bins) and, with
    ``write``, writes it one value per line to the file's
    ``*_dedisp_folded.txt`` (Fold_GPU::write_to_file).  ``overlap`` reads the
    file on a second thread into pinned buffers while the device works (the
    reads, their order and the result are the same either way); ``stats``
    receives the samples processed and the wall time."""
    from .dedisp import Dedisperser
    from .fold import Fold_GPU

    t0 = time.perf_counter()
    f = PSRDADA(filename)
    # band in MHz from the header, lower edge f0 = FREQ - BW/2, both in float
    bw = np.float32(f.bw)
    f0 = np.float32(np.float32(f.fc) - bw / np.float32(2))
    bw = float(np.float32(bw * np.float32(1e6)))
    f0 = float(np.float32(f0 * np.float32(1e6)))
    a = Dedisperser(bw, [dm], f0, fftpoint, count, precision=precision)
    b = Dedisperser(bw, [dm], f0, fftpoint, count, precision=precision)
    M = a.M
    f.initBuffer(count * M)
    fold = Fold_GPU(period, bw, count * M, time_bin=time_bin)
    fold.discard_samples(int(a.Nd[0]))
    first = True
    reads = 0
    for p1, p2 in _reads(f, overlap):
        reads += 1
        # blank data at the head of the file is skipped
        if first:
            if p1[0, 0] == 0:
                continue
            first = False
        a.filter_block(p1)
        b.filter_block(p2)
        fold.calculate_intensity(a, b)
        fold.fold_data()
    prof = fold.fold_data_bins()
    if stats is not None:
        stats.update(samples=reads * count * M, seconds=time.perf_counter() - t0, reads=reads)
    if write:
        with open(f.outfileName, "w") as out:
            for v in prof:
                out.write(f"{float(v):g}\n")
    f.close()
    a.close()
    b.close()
    return prof


def main() -> None:
    ap = argparse.ArgumentParser(description="dedisperse and fold a two-polarisation PSRDADA file")
    ap.add_argument("--file", required=True)
    ap.add_argument("--dm", type=float, default=750.0)
    ap.add_argument("--period", type=float, required=True)
    ap.add_argument("--fftpoint", type=int, default=2097152)
    ap.add_argument("--time-bin", type=int, default=1024)
    ap.add_argument("--count", type=int, default=1, help="FFT blocks per read")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--no-overlap", action="store_true", help="read the file on the calling thread")
    a = ap.parse_args()
    st = {}
    prof = fold_file(a.file, a.dm, a.period, a.fftpoint, a.count, a.time_bin, a.precision,
                     overlap=not a.no_overlap, stats=st)
    print(f"folded {prof.size} bins -> {os.path.splitext(a.file)[0]}_dedisp_folded.txt; "
          f"{st['samples']} samples per polarisation in {st['seconds']:.2f} s "
          f"({st['samples'] / st['seconds'] / 1e6:.1f} Msamples/s)")


if __name__ == "__main__":
    main()
