"""Filter design and segmentation through the C ABI (reference L3:
dedispersion/msosm/msosm_prepare.cpp, dedispersion/overlap_save/osm_prepare.cpp)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._abi import check, lib


def nd(bw: float, dm: float, f0: float) -> int:
    """Dispersion smear in samples (f0 = lower band edge, Hz)."""
    v = ctypes.c_ulong()
    check(lib().msosm_prepare_nd(bw, dm, f0, ctypes.byref(v)))
    return int(v.value)


def msosm_min_order(Nd: int) -> int:
    v = ctypes.c_ulong()
    check(lib().msosm_prepare_min_order_msosm(int(Nd), ctypes.byref(v)))
    return int(v.value)


def osm_min_order(Nd: int) -> int:
    v = ctypes.c_ulong()
    check(lib().msosm_prepare_min_order_osm(int(Nd), ctypes.byref(v)))
    return int(v.value)


def segmentation(bw: float, dm: float, f0: float, M: int):
    """(delaycount, delay_points[2M])."""
    out = np.zeros(2 * int(M), np.int32)
    dc = ctypes.c_int()
    check(lib().msosm_prepare_segmentation(bw, dm, f0, int(M), ctypes.byref(dc), out.ctypes.data))
    return int(dc.value), out


def dedisp_params(bw: float, dm: float, f0: float, M: int) -> np.ndarray:
    """H[2M] designed on the GPU in the reference's scaling."""
    out = np.zeros(2 * int(M), np.complex64)
    check(lib().msosm_prepare_dedisp_params(bw, dm, f0, int(M), out.ctypes.data))
    return out


class FoldPlanner:
    """Sample -> (period, phase) map of the Fold_GPU state machine as the
    device fold applies it (host only)."""

    def __init__(self, period: float, fs: float, discard_Nd: int = 0):
        h = ctypes.c_void_p()
        check(lib().msosm_fold_planner_create(period, fs, int(discard_Nd), ctypes.byref(h)))
        self._h = h

    def chunk(self, size: int):
        dest = np.zeros(int(size), np.int64)
        done = ctypes.c_ulonglong()
        check(lib().msosm_fold_planner_chunk(self._h, int(size), dest.ctypes.data, ctypes.byref(done)))
        return dest, int(done.value)

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().msosm_fold_planner_destroy(self._h)
            self._h = ctypes.c_void_p()
