"""Dedispersed series to a file while the device keeps working
(``msosm_writer_*``): the output-file threads of the reference's drivers
(multiple_dm_concurrent_msosm.cpp:80-146) without their busy-wait.

    with SeriesWriter(dedisperser, "out.bin") as w:
        for chunk in chunks:
            dedisperser.filter_block(chunk)
            w.push()

The file holds, per call, numDMs x count*M samples in the layout [dm][count*M]:
uint16 offset-binary pairs (``kind="uint16"``, the get_output codec) or
complex64 (``kind="c64"``).
"""
from __future__ import annotations

import ctypes
import datetime

from . import _abi
from ._abi import check, lib


def reference_file_name(num_dms: int, thread_id=None) -> str:
    """The reference writer's name: local time, then the trial count (and the
    thread id), '.bin' (multiple_dm_concurrent_msosm.cpp:84-99, 120-132)."""
    stamp = datetime.datetime.now().strftime("%Y-%m-%d %H:%M:%S")
    return f"{stamp}_{num_dms}" + ("" if thread_id is None else f"_{thread_id}") + ".bin"


class SeriesWriter:
    def __init__(self, dedisperser, path: str, kind: str = "uint16", depth: int = 2, threads: int = 1):
        k = {"uint16": _abi.WRITE_UINT16, "c64": _abi.WRITE_C64}[kind]
        h = ctypes.c_void_p()
        check(lib().msosm_writer_create(dedisperser._h, path.encode(), k, int(depth), int(threads),
                                        ctypes.byref(h)))
        self._h = h
        self._d = dedisperser  # keeps the handle alive while the writer is open
        self.path = path
        self.bytes_written = 0

    def push(self) -> None:
        """Queue the series of the handle's last filter call."""
        check(lib().msosm_writer_push(self._h))

    def close(self) -> int:
        if getattr(self, "_h", None) is not None and self._h.value:
            n = ctypes.c_ulonglong()
            h, self._h = self._h, None
            check(lib().msosm_writer_close(h, ctypes.byref(n)))
            self.bytes_written = int(n.value)
        return self.bytes_written

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
