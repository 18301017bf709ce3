"""msosm_gpu_b200 -- B200-native (sm_100a) coherent dedispersion.

MS-OSM / OSM dedispersion of complex baseband for many DM trials at once,
with fused detection and folding, behind a C ABI (include/msosm_b200.h)
implemented by the in-tree libmsosm_b200.so.  This package is the Python
face of that ABI; it has no compute path of its own.
"""
from ._abi import MsosmError, lib  # noqa: F401
from .fold import Fold_GPU  # noqa: F401
from .dedisp import (  # noqa: F401
    DedispBatch,
    Dedisperser,
    MSOSM_GPU_BATCH,
    MSOSM_GPU_DM_concurrent,
    OSM_GPU_BATCH,
    OSM_GPU_DM_concurrent,
)

__all__ = [
    "DedispBatch",
    "Dedisperser",
    "MSOSM_GPU_BATCH",
    "MSOSM_GPU_DM_concurrent",
    "OSM_GPU_BATCH",
    "OSM_GPU_DM_concurrent",
    "Fold_GPU",
    "MsosmError",
    "lib",
]
