"""Fold_GPU (folding/fold_gpu.cpp) over the C ABI: detection of one or two
polarisations and folding on the device."""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from ._abi import check, lib


class Fold_GPU:
    """Fold_GPU(period, fs, size, time_bin=-1): fold successive chunks of
    ``size`` samples.  calculate_intensity takes two Dedisperser objects (or
    raw device pointers) whose last output is the chunk (sqrt(|a|^2+|b|^2));
    set_intensity takes the intensities directly (host array or CUDA tensor)."""

    def __init__(self, period: float, fs: float, size: int, outfileName: str = "fold.txt", time_bin: int = -1):
        tb = (1 << 64) - 1 if time_bin is None or time_bin < 0 else int(time_bin)
        h = ctypes.c_void_p()
        check(lib().msosm_fold_create(float(period), float(fs), int(size), tb, ctypes.byref(h)))
        self._h = h
        self.size = int(size)
        self.outfileName = outfileName
        ps, tbo = ctypes.c_ulong(), ctypes.c_ulong()
        check(lib().msosm_fold_get_shape(self._h, ctypes.byref(ps), ctypes.byref(tbo)))
        self.period_samples = int(ps.value)
        self.time_bin = int(tbo.value)
        self.folded_data: Optional[np.ndarray] = None

    def discard_samples(self, Nd: int) -> None:
        check(lib().msosm_fold_discard_samples(self._h, int(Nd)))

    def calculate_intensity(self, pol1, pol2=None) -> None:
        handle = lambda p: getattr(p, "_h", None) if p is not None else None  # noqa: E731
        if hasattr(pol1, "output_device_ptr") and (pol2 is None or hasattr(pol2, "output_device_ptr")):
            check(lib().msosm_fold_calculate_intensity_dedisp(self._h, handle(pol1), handle(pol2)))
            return

        def ptr(p):
            if p is None:
                return None
            if hasattr(p, "output_device_ptr"):
                return ctypes.c_void_p(p.output_device_ptr())
            if hasattr(p, "data_ptr"):
                return ctypes.c_void_p(p.data_ptr())
            return ctypes.c_void_p(int(p))
        check(lib().msosm_fold_calculate_intensity(self._h, ptr(pol1), ptr(pol2)))

    def set_intensity(self, intensity) -> None:
        if hasattr(intensity, "data_ptr"):
            assert intensity.numel() == self.size and intensity.is_contiguous()
            if intensity.is_cuda:
                import torch
                torch.cuda.current_stream(intensity.device).synchronize()
            check(lib().msosm_fold_set_intensity(self._h, ctypes.c_void_p(intensity.data_ptr())))
            return
        a = np.ascontiguousarray(intensity, np.float32).reshape(-1)
        assert a.size == self.size
        check(lib().msosm_fold_set_intensity(self._h, a.ctypes.data))

    @property
    def total_intensity(self) -> np.ndarray:
        out = np.zeros(self.size, np.float32)
        check(lib().msosm_fold_get_intensity(self._h, out.ctypes.data))
        return out

    def fold_data(self) -> None:
        check(lib().msosm_fold_data(self._h))

    def fold_data_bins(self) -> np.ndarray:
        out = np.zeros(self.time_bin, np.float32)
        check(lib().msosm_fold_data_bins(self._h, out.ctypes.data))
        self.folded_data = out
        return out

    def write_to_file(self) -> None:
        with open(self.outfileName, "w") as f:
            for v in (self.folded_data if self.folded_data is not None else self.fold_data_bins()):
                f.write(f"{v:g}\n")

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().msosm_fold_destroy(self._h)
            self._h = ctypes.c_void_p()
