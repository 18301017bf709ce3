"""Build the in-tree shared library msosm_gpu_b200/libmsosm_b200.so (sm_100a).

    python -m msosm_gpu_b200.build [--force] [--verbose]

nvcc cross-compiles on a machine without a GPU.  The library links the CUDA
runtime statically, so it needs only the driver at run time.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libmsosm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(INCLUDE, "*.h")))


OBJDIR = os.path.join(PKG, "_build")
COMMON = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]


def _obj(src: str) -> str:
    return os.path.join(OBJDIR, os.path.basename(src) + ".o")


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile each source to an object (in parallel; a source is recompiled
    when it, any header or this script is newer than its object) and link
    the shared library with the CUDA runtime linked in statically."""
    if not force and not ptxas_verbose and up_to_date():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    newest_dep = max(os.path.getmtime(f) for f in headers() + [__file__])
    flags = (["-Xptxas", "-v"] if ptxas_verbose else []) + COMMON

    def stale(src: str) -> bool:
        o = _obj(src)
        return (force or ptxas_verbose or not os.path.exists(o)
                or os.path.getmtime(o) < max(os.path.getmtime(src), newest_dep))

    def compile_one(src: str):
        cmd = [nvcc(), *flags, "-c", src, "-o", _obj(src) + ".tmp"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            os.replace(_obj(src) + ".tmp", _obj(src))
        return src, r

    from concurrent.futures import ThreadPoolExecutor
    todo = [s for s in sources() if stale(s)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        results = list(ex.map(compile_one, todo))
    failed = [(s, r) for s, r in results if r.returncode != 0]
    for s, r in results:
        if r.returncode != 0 or ptxas_verbose or verbose:
            sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(os.path.basename(s) for s, _ in failed))
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *[_obj(s) for s in sources()]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed linking libmsosm_b200.so")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/smem usage")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))
