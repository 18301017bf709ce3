"""Python face of the C ABI: a DM-trial dedisperser plus classes named and
shaped like the reference's host API (dedispersion/include/*.h).

Host inputs are numpy arrays (complex64, or uint16 offset-binary pairs);
device inputs are CUDA tensors (torch) whose data pointer goes straight to
the kernels.  Every call goes through libmsosm_b200.so.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import check, lib


def _f32_array(v, n: Optional[int] = None) -> np.ndarray:
    a = np.ascontiguousarray(np.atleast_1d(np.asarray(v, dtype=np.float32)))
    if n is not None and a.size == 1 and n > 1:
        a = np.ascontiguousarray(np.full(n, a[0], np.float32))
    return a


def _input_pointer(x, n_samples: int):
    """(pointer, kind, keepalive) for a block of n_samples complex samples."""
    try:
        import torch
        if isinstance(x, torch.Tensor):
            if x.is_cuda:
                if x.dtype == torch.complex64:
                    kind = "c64"
                elif x.dtype in (torch.int32, torch.uint32 if hasattr(torch, "uint32") else torch.int32):
                    kind = "u16"
                elif x.dtype in (torch.int16, getattr(torch, "uint16", torch.int16)):
                    kind = "u16"
                else:
                    raise TypeError(f"unsupported tensor dtype {x.dtype}")
                if not x.is_contiguous():
                    raise ValueError("input tensor must be contiguous")
                nbytes = x.numel() * x.element_size()
                if nbytes != n_samples * (8 if kind == "c64" else 4):
                    raise ValueError(f"input holds {nbytes} bytes, expected {n_samples} samples")
                return x.data_ptr(), kind, x
            x = x.numpy()
    except ImportError:
        pass
    a = np.asarray(x)
    if a.dtype == np.complex64:
        kind, nbytes = "c64", 8
    elif a.dtype in (np.uint16, np.uint32):
        kind, nbytes = "u16", 4
    elif a.dtype == np.complex128:
        a = a.astype(np.complex64)
        kind, nbytes = "c64", 8
    else:
        raise TypeError(f"unsupported input dtype {a.dtype}: use complex64 or uint16 pairs")
    a = np.ascontiguousarray(a)
    if a.nbytes != n_samples * nbytes:
        raise ValueError(f"input holds {a.nbytes} bytes, expected {n_samples} samples")
    return a.ctypes.data, kind, a


class Dedisperser:
    """N DM trials over one complex baseband stream (msosm_dedisp handle).

    bw, f0: band width and LOWER band edge in Hz (scalars or per trial);
    dm: trial DMs.  fftpoint 0 picks the minimum; a smaller one is raised to
    the minimum like the reference does.  ``series`` materialises the
    dedispersed series (needed by get_output); ``osm`` selects classical
    overlap-save.  ``precision`` "fp32" (default) runs the inverse transforms
    on the CUDA cores in FP32; "fp16" / "bf16" run them on the tensor cores
    with f16 / bf16 operands and f32 accumulation (FFT sizes 4096, 8192 and
    16384).
    """

    def __init__(self, bw, dm, f0, fftpoint: int = 0, count: int = 1, input_size: int = 0,
                 osm: bool = False, series: bool = True, precision: str = "fp32"):
        if precision not in ("fp32", "fp16", "bf16"):
            raise ValueError("precision must be 'fp32', 'fp16' or 'bf16'")
        dm = _f32_array(dm)
        n = dm.size
        bw = _f32_array(bw, n)
        f0 = _f32_array(f0, n)
        if bw.size != n or f0.size != n:
            raise ValueError("bw, dm, f0 must be scalars or arrays of one length")
        self._params = (bw, dm, f0)
        flags = ((_abi.FLAG_OSM if osm else 0) | (0 if series else _abi.FLAG_NO_SERIES)
                 | (_abi.FLAG_TENSOR_F16 if precision == "fp16" else 0)
                 | (_abi.FLAG_TENSOR_BF16 if precision == "bf16" else 0))
        h = ctypes.c_void_p()
        check(lib().msosm_dedisp_create(bw.ctypes.data, dm.ctypes.data, f0.ctypes.data, n,
                                        int(fftpoint), int(count), int(input_size), flags,
                                        ctypes.byref(h)))
        self._h = h
        info = self.info()
        self.numDMs = n
        self.M = int(info.M)
        self.fftpoint = int(info.fftpoint)
        self.M_min = int(info.M_min)
        self.count = int(info.count)
        self.ring_slots = int(info.ring_slots)
        self.osm = osm
        self.series = series
        self.precision = precision
        nd = np.zeros(n, np.uint64)
        check(lib().msosm_dedisp_get_nd(self._h, nd.ctypes.data))
        self.Nd = nd
        dc = np.zeros(n, np.int32)
        check(lib().msosm_dedisp_get_delaycount(self._h, dc.ctypes.data))
        self.delaycount = dc
        self.folding = False

    # -- introspection --------------------------------------------------------
    def info(self) -> _abi.DedispInfo:
        inf = _abi.DedispInfo()
        check(lib().msosm_dedisp_get_info(self._h, ctypes.byref(inf)))
        return inf

    def delay_points(self, i: int) -> np.ndarray:
        out = np.zeros(self.fftpoint, np.int32)
        check(lib().msosm_dedisp_get_delay_points(self._h, int(i), out.ctypes.data))
        return out

    def dedisp_params(self, i: int) -> np.ndarray:
        out = np.zeros(self.fftpoint, np.complex64)
        check(lib().msosm_dedisp_get_dedisp_params(self._h, int(i), out.ctypes.data))
        return out

    @property
    def block_samples(self) -> int:
        return self.count * self.M

    # -- processing -------------------------------------------------------------
    def set_stream(self, stream) -> None:
        """Run on a CUDA stream (torch.cuda.Stream or a raw non-null
        cudaStream_t); None returns to the handle's own stream."""
        ptr = getattr(stream, "cuda_stream", stream) or 0
        check(lib().msosm_dedisp_set_stream(self._h, ctypes.c_void_p(ptr)))
        self._stream_ptr = ptr

    def set_tc_wait_limit(self, ns: int) -> None:
        """Limit of each wait of the tensor-core kernel on a GEMM, in ns
        (negative: the default 1 s; 0: every wait gives up at once).  A wait that gives up makes the next synchronising call raise
        a timeout; the handle then carries on.  For tests of that path."""
        check(lib().msosm_dedisp_set_tc_wait_limit(self._h, int(ns)))

    def filter_block(self, x) -> None:
        """Dedisperse the next count*M samples (host array or CUDA tensor)."""
        ptr, kind, keep = _input_pointer(x, self.block_samples)
        if not isinstance(keep, np.ndarray):
            # a CUDA tensor written on torch's current stream: make it ready
            # before the handle's stream reads it
            import torch
            cur = torch.cuda.current_stream(keep.device)
            if cur.cuda_stream != getattr(self, "_stream_ptr", 0) or cur.cuda_stream == 0:
                cur.synchronize()
        fn = lib().msosm_dedisp_filter_block_c64 if kind == "c64" else lib().msosm_dedisp_filter_block_uint16
        check(fn(self._h, ctypes.c_void_p(ptr)))
        del keep

    def get_output(self, out: Optional[np.ndarray] = None, dtype=np.complex64) -> np.ndarray:
        """Series of the last call, shape (numDMs, count*M) (complex64) or
        (numDMs, count*M, 2) uint16.  With ``out`` of numDMs*count*M + 1
        elements the reference layout (trailing zero element) is filled."""
        n = self.numDMs * self.block_samples + 1
        if dtype == np.complex64:
            buf = out if out is not None else np.zeros(n, np.complex64)
            assert buf.dtype == np.complex64 and buf.size == n and buf.flags.c_contiguous
            check(lib().msosm_dedisp_get_output_c64(self._h, buf.ctypes.data))
            return buf if out is not None else buf[:-1].reshape(self.numDMs, self.block_samples)
        buf = out if out is not None else np.zeros((n, 2), np.uint16)
        assert buf.dtype == np.uint16 and buf.size == 2 * n and buf.flags.c_contiguous
        check(lib().msosm_dedisp_get_output_uint16(self._h, buf.ctypes.data))
        return buf if out is not None else buf[:-1].reshape(self.numDMs, self.block_samples, 2)

    def output_device_ptr(self) -> int:
        p = ctypes.c_void_p()
        check(lib().msosm_dedisp_output_device_ptr(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    def fold_init(self, period: float, fs: float, time_bin: int = 0, discard_Nd: int = 0,
                  detect: str = "power") -> None:
        det = {"power": _abi.DETECT_POWER, "amplitude": _abi.DETECT_AMPLITUDE}[detect]
        check(lib().msosm_dedisp_fold_init(self._h, float(period), float(fs), int(time_bin),
                                           int(discard_Nd), det))
        ps = int(np.float32(period) * np.float32(fs))
        self.period_samples = ps
        self.time_bin = ps if time_bin == 0 else int(time_bin)
        self.folding = True

    def get_profiles(self) -> np.ndarray:
        out = np.zeros((self.numDMs, self.time_bin), np.float32)
        check(lib().msosm_dedisp_get_profiles(self._h, out.ctypes.data))
        return out

    def folded_periods(self) -> int:
        n = ctypes.c_ulonglong()
        check(lib().msosm_dedisp_folded_periods(self._h, ctypes.byref(n)))
        return int(n.value)

    def synchronize(self) -> None:
        check(lib().msosm_dedisp_synchronize(self._h))

    def reset(self) -> None:
        """Start a new input stream (same band and trials): the history is
        forgotten and folding unconfigured (call fold_init again)."""
        check(lib().msosm_dedisp_reset(self._h))
        self.folding = False

    def enable_timing(self, on: bool = True) -> None:
        """Record CUDA events around each stage of every filter call."""
        check(lib().msosm_dedisp_enable_timing(self._h, int(on)))

    def timing(self) -> dict:
        t = _abi.Timing()
        check(lib().msosm_dedisp_get_timing(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in _abi.Timing._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().msosm_dedisp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DedispBatch:
    """One filter call of many Dedisperser handles (observations of any
    length, band and trial grid) with one persistent launch per group of
    handles that run the same tensor-core kernel (msosm_batch): work items
    of every observation are handed out largest first from a counter.
    Handles of other kernels run their calls one after another inside the
    same call.  While in a batch the handles run on the batch's stream;
    read their results with their own get_output / get_profiles."""

    def __init__(self, dedispersers: Sequence[Dedisperser]):
        self.members = list(dedispersers)
        arr = (ctypes.c_void_p * len(self.members))(*[d._h.value for d in self.members])
        h = ctypes.c_void_p()
        check(lib().msosm_batch_create(arr, len(self.members), ctypes.byref(h)))
        self._h = h

    def info(self) -> dict:
        g, l, it = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().msosm_batch_get_info(self._h, ctypes.byref(g), ctypes.byref(l), ctypes.byref(it)))
        return {"groups": g.value, "launches_per_call": l.value, "items": it.value}

    def filter_block(self, inputs) -> None:
        """inputs[i]: the next count*M samples of member i (host arrays or
        CUDA tensors, all complex64 or all uint16 pairs)."""
        if len(inputs) != len(self.members):
            raise ValueError("one input per member")
        ptrs, kinds, keep = [], set(), []
        for d, x in zip(self.members, inputs):
            p, kind, k = _input_pointer(x, d.block_samples)
            ptrs.append(p)
            kinds.add(kind)
            keep.append(k)
            if not isinstance(k, np.ndarray):
                import torch
                torch.cuda.current_stream(k.device).synchronize()
        if len(kinds) != 1:
            raise ValueError("all inputs of a batch call must be of one kind")
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        kind = _abi.INPUT_C64 if kinds.pop() == "c64" else _abi.INPUT_UINT16
        check(lib().msosm_batch_filter(self._h, arr, kind))
        del keep

    def set_stream(self, stream) -> None:
        """Run on a CUDA stream (torch.cuda.Stream or a raw cudaStream_t);
        None returns to the batch's own stream."""
        ptr = getattr(stream, "cuda_stream", stream) or 0
        check(lib().msosm_batch_set_stream(self._h, ctypes.c_void_p(ptr)))

    def synchronize(self) -> None:
        check(lib().msosm_batch_synchronize(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().msosm_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# reference-shaped classes (dedispersion/include/*.h)
# ---------------------------------------------------------------------------

class MSOSM_GPU_DM_concurrent:
    """dedispersion/include/msosm_gpu_concurrent.h:15-64 over the C ABI."""

    def __init__(self, bw: Sequence[float], dm: Sequence[float], f0: Sequence[float], numDMs: int):
        self.numDMs = int(numDMs)
        self._bw = _f32_array(bw, self.numDMs)[: self.numDMs]
        self._dm = _f32_array(dm, self.numDMs)[: self.numDMs]
        self._f0 = _f32_array(f0, self.numDMs)[: self.numDMs]
        self._d: Optional[Dedisperser] = None
        self.wait_for_cpu = False

    def initialize_uint16(self, fftpoint: int, count: int = 1, input_size: int = 0,
                          compute_only: bool = False) -> None:
        self._d = Dedisperser(self._bw, self._dm, self._f0, fftpoint, count, input_size)
        self.count = self._d.count
        self.M_common = self._d.M
        self.M_common_min = self._d.M_min
        self.Nd = self._d.Nd
        self.delaycount = self._d.delaycount
        self.compute_only = compute_only

    def filter_block_uint16(self, input) -> None:
        self._d.filter_block(input)

    def get_output(self, output: np.ndarray) -> None:
        self._d.get_output(out=output, dtype=output.dtype.type if output.dtype == np.uint16 else np.complex64)

    def synchronize(self) -> None:
        self._d.synchronize()

    def reset_device(self) -> None:
        # the reference calls cudaDeviceReset, which ends every allocation of
        # the process; here only this object's resources are released
        if self._d is not None:
            self._d.close()

    @property
    def delay_points(self):
        return [self._d.delay_points(i) for i in range(self.numDMs)]

    @property
    def dedisp_params(self):
        return [self._d.dedisp_params(i) for i in range(self.numDMs)]


class MSOSM_GPU_BATCH:
    """dedispersion/include/msosm_gpu_batch.h:7-41 (one DM) over the C ABI."""

    def __init__(self, bw: float = 0, dm: float = 0, f0: float = 0):
        self._p = (float(bw), float(dm), float(f0))
        self._d: Optional[Dedisperser] = None

    def initialize_uint16(self, fftpoint: int = 0, count: int = 1) -> None:
        bw, dm, f0 = self._p
        self._d = Dedisperser(bw, dm, f0, fftpoint, count)
        self.count = self._d.count
        self.M = self._d.M
        self.M_min = self._d.M_min
        self.Nd = int(self._d.Nd[0])
        self.delaycount = int(self._d.delaycount[0])
        self.delay_points = self._d.delay_points(0)
        self.dedisp_params = self._d.dedisp_params(0)

    def filter_block_uint16(self, input) -> None:
        self._d.filter_block(input)

    def get_output(self, output: Optional[np.ndarray] = None) -> np.ndarray:
        res = self._d.get_output()
        if output is not None:
            output.reshape(-1)[: res.size] = res.reshape(-1)
            return output
        return res.reshape(-1)

    @property
    def output_buffer_d(self) -> int:
        return self._d.output_device_ptr()


class OSM_GPU_BATCH(MSOSM_GPU_BATCH):
    """dedispersion/include/osm_gpu_batch.h:7-37: classical overlap-save."""

    def initialize_uint16(self, fftpoint: int = 0, count: int = 1, streaming: bool = False) -> None:
        bw, dm, f0 = self._p
        self._d = Dedisperser(bw, dm, f0, fftpoint, count, osm=True)
        self.count = self._d.count
        self.M = self._d.M
        self.M_min = self._d.M_min
        self.Nd = int(self._d.Nd[0])
        self.dedisp_params = self._d.dedisp_params(0)


class OSM_GPU_DM_concurrent(MSOSM_GPU_DM_concurrent):
    """dedispersion/include/osm_gpu_concurrent.h:7-42."""

    def initialize_uint16(self, fftpoint: int = 0, count: int = 1, compute_only: bool = False) -> None:
        self._d = Dedisperser(self._bw, self._dm, self._f0, fftpoint, count, osm=True)
        self.count = self._d.count
        self.M_common = self._d.M
        self.M_common_min = self._d.M_min
        self.Nd = self._d.Nd
        self.compute_only = compute_only


def tc_gemm_check(step: int, a: np.ndarray) -> np.ndarray:
    """Run GEMM ``step`` of the tensor-core kernel on a float16 matrix ``a``
    with the kernel's own layouts (msosm_tc_gemm_check): steps 1, 2 the
    4096-point GEMMs (a 128 x 128; result 128 x 128 / 128 x 64), step 3 the
    8192- and 16384-point GEMM 1 (a 128 x 256; result 128 x 256), step 4 the
    16384-point GEMM 2 (a 128 x 256; result 128 x 128).  Returns a @ B_step
    as float32."""
    a = np.ascontiguousarray(a, dtype=np.float16)
    kdim = 256 if step >= 3 else 128
    if a.shape != (128, kdim):
        raise ValueError(f"a must be 128 x {kdim}")
    d = np.zeros((128, {1: 128, 2: 64, 3: 256, 4: 128}[step]), np.float32)
    check(lib().msosm_tc_gemm_check(int(step), a.view(np.uint16).ctypes.data, d.ctypes.data))
    return d
