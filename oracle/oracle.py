"""ctypes view of the FP64 C restatement (oracle/orc.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline leg, always as the checker.  The product
package ``msosm_gpu_b200`` never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
from typing import Dict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liborc.so")
REF_GOLDEN = os.path.join(HERE, "_ref", "ref_golden")
REF_GPU_RUNNER = os.path.join(HERE, "_ref", "ref_gpu_runner")


def reference_checkout() -> str | None:
    """The msosm_gpu source tree the reference-side checkers are built from:
    $MSOSM_REFERENCE, else a `reference` directory beside this repository;
    None when neither holds the reference's sources."""
    root = os.path.dirname(HERE)
    for p in (os.environ.get("MSOSM_REFERENCE"), os.path.join(os.path.dirname(root), "reference")):
        if p and os.path.isfile(os.path.join(p, "gpu", "gpu_kernel.cu")):
            return p
    return None

_lib = None


def build() -> None:
    """Compile liborc.so (gcc, seconds)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        f32, u64, i32, dp = ctypes.c_float, ctypes.c_ulong, ctypes.c_int, ctypes.c_void_p
        sig = {
            "orc_nd": (u64, [f32, f32, f32]),
            "orc_msosm_min_order": (u64, [u64]),
            "orc_osm_min_order": (u64, [u64]),
            "orc_delaycount": (i32, [u64, u64]),
            "orc_segmentation": (i32, [f32, f32, f32, u64, u64, dp]),
            "orc_dedisp_params": (None, [f32, f32, f32, u64, i32, dp]),
            "orc_chirp_phase": (ctypes.c_double, [f32, f32, f32, u64, u64]),
            "orc_fft": (None, [dp, u64, i32]),
            "orc_decode_uint16": (None, [dp, ctypes.c_size_t, dp]),
            "orc_encode_uint16": (None, [dp, ctypes.c_size_t, dp]),
            "orc_dedisp_create": (dp, [dp, dp, dp, i32, u64, i32, u64, i32, i32]),
            "orc_dedisp_destroy": (None, [dp]),
            "orc_dedisp_M": (u64, [dp]),
            "orc_dedisp_count": (i32, [dp]),
            "orc_dedisp_ring_slots": (i32, [dp]),
            "orc_dedisp_delaycount": (i32, [dp, i32]),
            "orc_dedisp_Nd": (u64, [dp, i32]),
            "orc_dedisp_filter": (None, [dp, dp, dp]),
            "orc_intensity": (None, [dp, dp, ctypes.c_size_t, dp]),
            "orc_fold_create": (dp, [f32, f32, u64, u64, i32]),
            "orc_fold_destroy": (None, [dp]),
            "orc_fold_discard_samples": (None, [dp, u64]),
            "orc_fold_data": (None, [dp, dp]),
            "orc_fold_period_samples": (u64, [dp]),
            "orc_fold_time_bin": (u64, [dp]),
            "orc_fold_data_bins": (None, [dp, dp]),
            "orc_fold_period_starts": (ctypes.c_size_t, [f32, f32, u64, dp, ctypes.c_size_t]),
            "orc_simulate_two_spike": (u64, [f32, f32, f32, f32, u64, dp, u64]),
            "orc_set_threads": (None, [i32]),
            "orc_get_threads": (i32, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def nd(bw: float, dm: float, f0: float) -> int:
    return int(lib().orc_nd(bw, dm, f0))


def msosm_min_order(Nd: int) -> int:
    return int(lib().orc_msosm_min_order(Nd))


def osm_min_order(Nd: int) -> int:
    return int(lib().orc_osm_min_order(Nd))


def segmentation(bw: float, dm: float, f0: float, M: int):
    Nd = nd(bw, dm, f0)
    out = np.zeros(2 * M, np.int32)
    dc = lib().orc_segmentation(bw, dm, f0, Nd, M, _p(out))
    return dc, out


def dedisp_params(bw: float, dm: float, f0: float, M: int, sign: int = -1) -> np.ndarray:
    H = np.zeros(4 * M, np.float64)
    lib().orc_dedisp_params(bw, dm, f0, M, sign, _p(H))
    return H.view(np.complex128)


def decode_uint16(u16: np.ndarray) -> np.ndarray:
    u16 = np.ascontiguousarray(u16, np.uint16).reshape(-1)
    out = np.zeros(u16.size, np.float64)
    lib().orc_decode_uint16(_p(u16), u16.size // 2, _p(out))
    return out.view(np.complex128)


class Dedisp:
    """MSOSM_GPU_DM_concurrent / OSM_GPU_DM_concurrent semantics in FP64."""

    def __init__(self, bw, dm, f0, fftpoint, count=1, input_size=0, osm=False, threads=0):
        dm = np.ascontiguousarray(np.atleast_1d(dm), np.float32)
        n = dm.size
        bw = np.ascontiguousarray(np.broadcast_to(np.float32(bw), (n,)), np.float32)
        f0 = np.ascontiguousarray(np.broadcast_to(np.float32(f0), (n,)), np.float32)
        self._keep = (bw, dm, f0)
        self.h = lib().orc_dedisp_create(_p(bw), _p(dm), _p(f0), n, fftpoint, count,
                                         input_size, int(osm), threads)
        if not self.h:
            raise ValueError("oracle dedisperser rejected its parameters")
        self.numDMs = n
        self.M = int(lib().orc_dedisp_M(self.h))
        self.count = int(lib().orc_dedisp_count(self.h))
        self.ring_slots = int(lib().orc_dedisp_ring_slots(self.h))
        self.delaycount = [int(lib().orc_dedisp_delaycount(self.h, i)) for i in range(n)]
        self.Nd = [int(lib().orc_dedisp_Nd(self.h, i)) for i in range(n)]

    def filter(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.complex128).reshape(-1)
        assert x.size == self.count * self.M
        out = np.zeros(self.numDMs * self.count * self.M, np.complex128)
        lib().orc_dedisp_filter(self.h, _p(x), _p(out))
        return out.reshape(self.numDMs, self.count * self.M)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_dedisp_destroy(self.h)
            self.h = None


class Fold:
    """Fold_GPU state machine (folding/fold_gpu.cpp) in FP64 or float."""

    def __init__(self, period, fs, size, time_bin=-1, accumulate_float=False):
        tb = (1 << 64) - 1 if time_bin is None or time_bin < 0 else int(time_bin)
        self.size = int(size)
        self.h = lib().orc_fold_create(period, fs, size, tb, int(accumulate_float))
        self.period_samples = int(lib().orc_fold_period_samples(self.h))
        self.time_bin = int(lib().orc_fold_time_bin(self.h))

    def discard_samples(self, Nd: int):
        lib().orc_fold_discard_samples(self.h, int(Nd))

    def fold_data(self, intensity: np.ndarray):
        I = np.ascontiguousarray(intensity, np.float64).reshape(-1)
        assert I.size == self.size
        lib().orc_fold_data(self.h, _p(I))

    def fold_data_bins(self) -> np.ndarray:
        out = np.zeros(self.time_bin, np.float64)
        lib().orc_fold_data_bins(self.h, _p(out))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_fold_destroy(self.h)
            self.h = None


def intensity(a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, np.complex128).reshape(-1)
    out = np.zeros(a.size, np.float64)
    bp = None
    if b is not None:
        b = np.ascontiguousarray(b, np.complex128).reshape(-1)
        bp = _p(b)
    lib().orc_intensity(_p(a), bp, a.size, _p(out))
    return out


def period_starts(period: float, fs: float, total: int, cap: int = 1 << 20) -> np.ndarray:
    out = np.zeros(cap, np.int64)
    n = lib().orc_fold_period_starts(period, fs, total, _p(out), cap)
    return out[:n].copy()


def simulate_two_spike(bw, dm, f0, period, repeat=1) -> np.ndarray:
    Np = int(np.float32(period) * np.float32(bw))
    out = np.zeros(2 * Np * repeat, np.float64)
    got = lib().orc_simulate_two_spike(bw, dm, f0, period, repeat, _p(out), Np * repeat)
    if got == 0:
        raise ValueError("simulate_two_spike rejected its parameters")
    return out.view(np.complex128)


# ---------------------------------------------------------------------------
# record files written by ref_golden / ref_gpu_runner
# ---------------------------------------------------------------------------

_DT = {"u8": np.uint64, "i4": np.int32, "f4": np.float32, "f8": np.float64,
       "u2": np.uint16, "i8": np.int64}


def read_records(path: str) -> Dict[str, np.ndarray]:
    out = {}
    with open(path, "rb") as f:
        while True:
            hdr = f.read(48)
            if len(hdr) < 48:
                break
            name = hdr[:32].split(b"\0")[0].decode()
            dt = _DT[hdr[32:40].split(b"\0")[0].decode()]
            (count,) = struct.unpack("<Q", hdr[40:48])
            data = np.frombuffer(f.read(count * np.dtype(dt).itemsize), dtype=dt)
            out[name] = data.copy()
    return out
