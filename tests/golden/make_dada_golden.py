"""Regenerate tests/golden/reference_dada.json: what the reference's own
PSRDADA reader (psrdada/psrdada.cpp, compiled from its sources into
oracle/_ref/ref_golden) reads from seeded synthetic PSRDADA files -- header
fields, readCount, and a SHA-256 of the de-interleaved polarisations.  The
test (tests/test_psrdada_cpu.py) rebuilds the same files from the recorded
header text and seed and checks this library's reader against it.

    python tests/golden/make_dada_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

CASES = [
    # header text, seed, body uint16 pairs (both pols, interleaved frames), trailing bytes, n, reads
    {"header": "HDR_VERSION 1.0\nHDR_SIZE 4096\nBW 16\nFREQ 1250\nNBIT 16\nNCHAN 1\nNDIM 2\nNPOL 2\n",
     "seed": 1, "pairs": 3 * 2 * 2048, "trailing": 0, "n": 2048, "reads": 3},
    {"header": "HDR_VERSION 1.0\nBW 64.0\nFREQ    1400.5   # centre\nNBIT 8\nNCHAN\t4\nNDIM 2\n NPOL 1\n"
               "TELESCOPE Parkes\nNPOL 2\n",
     "seed": 2, "pairs": 5 * 2 * 2048, "trailing": 100, "n": 4096, "reads": 2,
     # "NCHAN\t4" has no space: the reference never sets nchan (left uninitialised)
     "absent": ["nchan"]},
]


def file_bytes(case) -> bytes:
    """The synthetic file of a case (the test builds it the same way)."""
    rng = np.random.default_rng(case["seed"])
    hdr = case["header"].encode()
    body = rng.integers(0, 65536, size=2 * case["pairs"], dtype=np.uint16).tobytes()
    tail = rng.integers(0, 256, size=case["trailing"], dtype=np.uint8).tobytes()
    return hdr + b"\0" * (4096 - len(hdr)) + body + tail


def main() -> None:
    ref = O.reference_checkout()
    if not ref:
        sys.exit("set MSOSM_REFERENCE to the msosm_gpu source tree")
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "golden", f"REF={ref}"], check=True)
    out = []
    with tempfile.TemporaryDirectory() as td:
        for i, c in enumerate(CASES):
            path, rec = os.path.join(td, f"case{i}.dada"), os.path.join(td, f"case{i}.rec")
            with open(path, "wb") as f:
                f.write(file_bytes(c))
            subprocess.run([O.REF_GOLDEN, "dada", path, str(c["n"]), str(c["reads"]), rec], check=True,
                           stdout=subprocess.DEVNULL)
            r = O.read_records(rec)
            ints = dict(zip(["nbit", "nchan", "ndim", "npol"], [int(v) for v in r["nbit_nchan_ndim_npol"]]))
            for k in c.get("absent", []):
                ints[k] = None
            out.append(dict(c, expected={
                "bw": float(r["bw_fc"][0]), "fc": float(r["bw_fc"][1]), **ints,
                "filesize": int(r["filesize"][0]), "readCount": int(r["readCount"][0]),
                "frameCount": int(r["frameCount"][0]),
                "pol1_sha256": hashlib.sha256(r["pol1"].astype(np.uint16).tobytes()).hexdigest(),
                "pol2_sha256": hashlib.sha256(r["pol2"].astype(np.uint16).tobytes()).hexdigest()}))
    with open(os.path.join(HERE, "reference_dada.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
