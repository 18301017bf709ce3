"""The reference's own driver programs (its 16 top-level .cpp files) compile
UNMODIFIED against this library's drop-in headers: include/compat/ gives the
reference's include names (globals.h, msosm_gpu_concurrent.h,
msosm_gpu_batch.h, osm_gpu_batch.h, fold_gpu.h, simulated_complex_signal.h,
...) over include/msosm_gpu_b200.hpp.  Needs the reference checkout
($MSOSM_REFERENCE, or `reference` beside this repository); skipped without
it.  tests/test_gpu_reference_drivers.py runs the prebuilt binaries."""
import glob
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = O.reference_checkout()


@pytest.mark.skipif(REF is None, reason="reference checkout not available")
def test_every_reference_driver_compiles_unchanged():
    drivers = sorted(glob.glob(os.path.join(REF, "*.cpp")))
    assert len(drivers) >= 16

    def compile_one(src):
        r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-I", os.path.join(ROOT, "include", "compat"),
                            "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", src],
                           capture_output=True, text=True)
        return os.path.basename(src), r.returncode, r.stderr[-1500:]

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(compile_one, drivers))
    bad = [(n, e) for n, rc, e in results if rc != 0]
    assert not bad, bad


def test_compat_headers_cover_the_reference_include_names():
    names = {"globals.h", "matplotlibcpp.h", "msosm_gpu_concurrent.h", "msosm_gpu_batch.h",
             "msosm_gpu_batch_stream.h", "osm_gpu_batch.h", "osm_gpu_concurrent.h", "prepare.h",
             "prepare_concurrent.h", "fold_gpu.h", "simulated_complex_signal.h", "AWGN.h", "psrdada.h"}
    have = {os.path.basename(p) for p in glob.glob(os.path.join(ROOT, "include", "compat", "*.h"))}
    assert names <= have, names - have
