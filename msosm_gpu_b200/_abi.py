"""ctypes binding of the C ABI in include/msosm_b200.h.

Loads the in-tree ``libmsosm_b200.so`` and fails loudly when it is missing:
there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmsosm_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "msosm_b200.h")

OK = 0
ERR_BAD_ARG = 1
ERR_OOM = 2
ERR_CUDA = 3
ERR_TIMEOUT = 4
ERR_UNSUPPORTED = 5
ERR_STATE = 6
ERR_NO_DEVICE = 7

FLAG_OSM = 0x1
FLAG_NO_SERIES = 0x2
FLAG_TENSOR_F16 = 0x4
FLAG_TENSOR_BF16 = 0x8
FLAG_DISPERSE = 0x10
WRITE_UINT16 = 0
WRITE_C64 = 1
SIM_TAG_PULSAR = 0
SIM_TAG_AWGN = 1
DETECT_POWER = 0
DETECT_AMPLITUDE = 1
INPUT_UINT16 = 0
INPUT_C64 = 1


class MsosmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[msosm status {status}] {msg}")
        self.status = status


class DedispInfo(ctypes.Structure):
    _fields_ = [
        ("M", ctypes.c_ulong),
        ("fftpoint", ctypes.c_ulong),
        ("M_min", ctypes.c_ulong),
        ("count", ctypes.c_int),
        ("numDMs", ctypes.c_int),
        ("ring_slots", ctypes.c_int),
        ("max_delaycount", ctypes.c_int),
        ("flags", ctypes.c_uint),
        ("calls", ctypes.c_ulonglong),
        ("device_bytes", ctypes.c_ulonglong),
    ]


class Timing(ctypes.Structure):
    _fields_ = [
        ("forward_ms", ctypes.c_double),
        ("dedisp_ms", ctypes.c_double),
        ("fold_ms", ctypes.c_double),
        ("h2d_ms", ctypes.c_double),
        ("calls", ctypes.c_ulonglong),
        ("kernel_launches", ctypes.c_ulonglong),
    ]


class SimTwoSpikeInfo(ctypes.Structure):
    _fields_ = [("Np", ctypes.c_ulong), ("Nd", ctypes.c_ulong), ("range", ctypes.c_ulong), ("order", ctypes.c_ulong)]


class SimPulsarParams(ctypes.Structure):
    _fields_ = [
        ("bw", ctypes.c_float),
        ("f0", ctypes.c_float),
        ("dm", ctypes.c_float),
        ("period", ctypes.c_double),
        ("fwhm", ctypes.c_double),
        ("centre", ctypes.c_double),
        ("snr", ctypes.c_double),
        ("seed", ctypes.c_ulonglong),
    ]


class SimPulsarInfo(ctypes.Structure):
    _fields_ = [("chunk", ctypes.c_ulong), ("M", ctypes.c_ulong), ("Nd", ctypes.c_ulong),
                ("next_sample", ctypes.c_ulonglong)]


class CnnConfig(ctypes.Structure):
    _fields_ = [("in_channels", ctypes.c_int), ("length", ctypes.c_int), ("channels", ctypes.c_int),
                ("kernel", ctypes.c_int), ("layers", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("dm_weight", ctypes.c_float)]


_lib = None


def _declare(L: ctypes.CDLL) -> None:
    f32, ul, i32, u32, vp = ctypes.c_float, ctypes.c_ulong, ctypes.c_int, ctypes.c_uint, ctypes.c_void_p
    pul, pi, pvp = ctypes.POINTER(ul), ctypes.POINTER(i32), ctypes.POINTER(vp)
    ull = ctypes.c_ulonglong
    pull = ctypes.POINTER(ull)
    sig = {
        "msosm_last_error": (ctypes.c_char_p, []),
        "msosm_version": (i32, []),
        "msosm_device_count": (i32, []),
        "msosm_prepare_nd": (i32, [f32, f32, f32, pul]),
        "msosm_prepare_min_order_msosm": (i32, [ul, pul]),
        "msosm_prepare_min_order_osm": (i32, [ul, pul]),
        "msosm_prepare_segmentation": (i32, [f32, f32, f32, ul, pi, vp]),
        "msosm_prepare_dedisp_params": (i32, [f32, f32, f32, ul, vp]),
        "msosm_prepare_dedisp_params_noalloc": (i32, [f32, f32, f32, ul, vp, vp]),
        "msosm_dedisp_create": (i32, [vp, vp, vp, i32, ul, i32, ul, u32, pvp]),
        "msosm_dedisp_destroy": (i32, [vp]),
        "msosm_dedisp_get_info": (i32, [vp, ctypes.POINTER(DedispInfo)]),
        "msosm_dedisp_get_nd": (i32, [vp, vp]),
        "msosm_dedisp_get_delaycount": (i32, [vp, vp]),
        "msosm_dedisp_get_delay_points": (i32, [vp, i32, vp]),
        "msosm_dedisp_get_dedisp_params": (i32, [vp, i32, vp]),
        "msosm_dedisp_set_stream": (i32, [vp, vp]),
        "msosm_dedisp_set_tc_wait_limit": (i32, [vp, ctypes.c_longlong]),
        "msosm_dedisp_reset": (i32, [vp]),
        "msosm_batch_create": (i32, [vp, i32, pvp]),
        "msosm_batch_destroy": (i32, [vp]),
        "msosm_batch_filter": (i32, [vp, vp, i32]),
        "msosm_batch_synchronize": (i32, [vp]),
        "msosm_batch_set_stream": (i32, [vp, vp]),
        "msosm_batch_get_info": (i32, [vp, pi, pi, pi]),
        "msosm_dedisp_filter_block_uint16": (i32, [vp, vp]),
        "msosm_dedisp_filter_block_c64": (i32, [vp, vp]),
        "msosm_dedisp_get_output_c64": (i32, [vp, vp]),
        "msosm_dedisp_get_output_uint16": (i32, [vp, vp]),
        "msosm_dedisp_output_device_ptr": (i32, [vp, pvp]),
        "msosm_dedisp_fold_init": (i32, [vp, f32, f32, ul, ul, i32]),
        "msosm_dedisp_get_profiles": (i32, [vp, vp]),
        "msosm_dedisp_folded_periods": (i32, [vp, pull]),
        "msosm_dedisp_synchronize": (i32, [vp]),
        "msosm_dedisp_enable_timing": (i32, [vp, i32]),
        "msosm_dedisp_get_timing": (i32, [vp, ctypes.POINTER(Timing)]),
        "msosm_fold_create": (i32, [f32, f32, ul, ul, pvp]),
        "msosm_fold_destroy": (i32, [vp]),
        "msosm_fold_discard_samples": (i32, [vp, ul]),
        "msosm_fold_calculate_intensity": (i32, [vp, vp, vp]),
        "msosm_fold_calculate_intensity_dedisp": (i32, [vp, vp, vp]),
        "msosm_fold_set_intensity": (i32, [vp, vp]),
        "msosm_fold_get_intensity": (i32, [vp, vp]),
        "msosm_fold_data": (i32, [vp]),
        "msosm_fold_data_bins": (i32, [vp, vp]),
        "msosm_fold_get_shape": (i32, [vp, pul, pul]),
        "msosm_fold_planner_create": (i32, [f32, f32, ul, pvp]),
        "msosm_fold_planner_destroy": (i32, [vp]),
        "msosm_fold_planner_chunk": (i32, [vp, ul, vp, pull]),
        "msosm_tc_gemm_check": (i32, [i32, vp, vp]),
        "msosm_dada_open": (i32, [ctypes.c_char_p, pvp]),
        "msosm_dada_close": (i32, [vp]),
        "msosm_dada_get_info": (i32, [vp, vp]),
        "msosm_dada_get_header": (i32, [vp, vp]),
        "msosm_dada_read_count": (i32, [vp, ul, pul]),
        "msosm_dada_read": (i32, [vp, ul, vp, vp]),
        "msosm_writer_create": (i32, [vp, ctypes.c_char_p, i32, i32, i32, pvp]),
        "msosm_writer_push": (i32, [vp]),
        "msosm_writer_close": (i32, [vp, pull]),
        "msosm_cnn_create": (i32, [ctypes.POINTER(CnnConfig), ull, pvp]),
        "msosm_cnn_destroy": (i32, [vp]),
        "msosm_cnn_param_count": (i32, [vp, ctypes.POINTER(ctypes.c_size_t)]),
        "msosm_cnn_get_params": (i32, [vp, vp]),
        "msosm_cnn_set_params": (i32, [vp, vp]),
        "msosm_cnn_forward": (i32, [vp, vp, i32, vp, vp]),
        "msosm_cnn_gradient": (i32, [vp, vp, vp, vp, i32, ctypes.POINTER(f32), vp]),
        "msosm_cnn_adam_step": (i32, [vp, f32]),
        "msosm_host_alloc": (i32, [ctypes.c_size_t, i32, pvp]),
        "msosm_host_free": (i32, [vp, i32]),
        "msosm_sim_normals": (i32, [ull, ull, ul, u32, vp, vp]),
        "msosm_sim_awgn": (i32, [ull, ul, i32, f32, f32, f32, vp]),
        "msosm_sim_two_spike_shape": (i32, [f32, f32, f32, f32, ctypes.POINTER(SimTwoSpikeInfo)]),
        "msosm_sim_two_spike": (i32, [f32, f32, f32, f32, ul, i32, f32, ull, vp, vp, ctypes.POINTER(f32)]),
        "msosm_sim_pulsar_create": (i32, [ctypes.POINTER(SimPulsarParams), ul, pvp]),
        "msosm_sim_pulsar_destroy": (i32, [vp]),
        "msosm_sim_pulsar_get_info": (i32, [vp, ctypes.POINTER(SimPulsarInfo)]),
        "msosm_sim_pulsar_next": (i32, [vp, vp, vp, ctypes.c_double]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def lib() -> ctypes.CDLL:
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m msosm_gpu_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise MsosmError(status, lib().msosm_last_error().decode(errors="replace"))


def header_functions() -> list:
    """Names of the functions declared in include/msosm_b200.h."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(msosm_[a-z0-9_]+)\s*\(", src)))
