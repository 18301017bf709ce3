"""Regenerate the golden fixtures in this directory from the reference itself.

Builds ``oracle/_ref/ref_golden`` (the reference's own host sources --
filter design, segmentation, Fold_GPU, SimulatedComplexSignal -- compiled in
place from the reference tree with the stand-in headers in oracle/ref_shim/)
and records what it computes.  Needs the reference checkout, so it runs on
the development machine only; the fixtures it writes are committed and the
tests read them anywhere.

    python tests/golden/make_golden.py [--ref /path/to/reference]
"""
from __future__ import annotations

import argparse
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

# (bw Hz, dm, f0 Hz = lower band edge, fftpoint); fftpoint 0 = minimum order
MSOSM_SETS = [
    (16e6, 50.0, 1242e6, 4096),    # 16 MHz at 1250 MHz centre, DM 50, FFT 4096
    (16e6, 73.2, 1242e6, 4096),    # same band, DM 73.2
    (16e6, 5.0, 1242e6, 1024),
    (16e6, 0.8, 1242e6, 0),        # minimum filter order
    (16e6, 30.0, 1242e6, 512),     # below the minimum: bumped to 2*M_min
    (64e6, 37.5, 1368e6, 8192),    # 64 MHz at 1400 MHz centre
    (4e6, 300.0, 1098e6, 2048),    # narrow band, high DM
    (32e6, 12.5, 1384e6, 2048),
]
# 256-trial grid over 0-100 at 16 MHz / 1242 MHz, FFT 4096: a subset of trials
CONCURRENT = (16e6, 1242e6, 4096, [100.0 * i / 255 for i in (1, 2, 17, 64, 128, 187, 255)])
OSM_SETS = [
    (16e6, 0.5, 1242e6, 0),
    (16e6, 0.25, 1242e6, 4096),
]
# (period s, fs Hz, chunk size, time_bin (-1 = none), Nd, chunks, seed)
FOLD_SETS = [
    (0.01234, 1e4, 1000, 10, 300, 20, 1),
    (0.01234, 1e4, 97, -1, 300, 60, 2),
    (0.00531, 2e4, 512, 7, 1000, 40, 3),
    (0.0031, 16e4, 2048, 16, 900, 30, 4),
    (0.0037, 2.5e5, 4096, 32, 5000, 12, 5),
]
SIM = (16e6, 5.0, 1242e6, 0.0005, 2)


def run(args):
    subprocess.run([O.REF_GOLDEN] + [str(a) for a in args], check=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=O.reference_checkout(),
                    help="the msosm_gpu source tree (default: $MSOSM_REFERENCE, or `reference` beside the repo)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("give --ref or set MSOSM_REFERENCE to the msosm_gpu source tree")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "golden", f"REF={a.ref}"], check=True)
    meta = {"generator": "tests/golden/make_golden.py", "msosm": [], "osm": [], "fold": []}
    arrays = {}
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "r.bin")
        for k, (bw, dm, f0, fp) in enumerate(MSOSM_SETS):
            run(["msosm", bw, dm, f0, fp, out])
            r = O.read_records(out)
            meta["msosm"].append({"bw": bw, "dm": dm, "f0": f0, "fftpoint": fp,
                                  "Nd": int(r["Nd"][0]), "M_min": int(r["M_min"][0]),
                                  "M": int(r["M"][0]), "delaycount": int(r["delaycount"][0])})
            arrays[f"msosm{k}_delay_points"] = r["delay_points"].astype(np.int16)
            arrays[f"msosm{k}_H"] = r["H"]
        bw, f0, fp, dms = CONCURRENT
        run(["concurrent", bw, f0, fp, out] + dms)
        r = O.read_records(out)
        meta["concurrent"] = {"bw": bw, "f0": f0, "fftpoint": fp, "dm": dms,
                              "M_common": int(r["M_common"][0]),
                              "M_common_min": int(r["M_common_min"][0]),
                              "Nd": r["Nd"].tolist(), "M_min": r["M_min"].tolist(),
                              "delaycount": r["delaycount"].tolist()}
        arrays["concurrent_delay_points"] = r["delay_points"].astype(np.int16)
        arrays["concurrent_H"] = r["H"]
        for k, (bw, dm, f0, fp) in enumerate(OSM_SETS):
            run(["osm", bw, dm, f0, fp, out])
            r = O.read_records(out)
            meta["osm"].append({"bw": bw, "dm": dm, "f0": f0, "fftpoint": fp,
                                "Nd": int(r["Nd"][0]), "M_min": int(r["M_min"][0]),
                                "M": int(r["M"][0])})
            arrays[f"osm{k}_H"] = r["H"]
        for k, (period, fs, size, tb, Nd, nch, seed) in enumerate(FOLD_SETS):
            rng = np.random.default_rng(seed)
            I = rng.integers(0, 50, size=size * nch).astype(np.uint8)
            inp = os.path.join(td, "I.f32")
            I.astype(np.float32).tofile(inp)
            run(["fold", period, fs, size, tb, Nd, nch, inp, out])
            r = O.read_records(out)
            meta["fold"].append({"period": period, "fs": fs, "size": size, "time_bin": tb,
                                 "Nd": Nd, "chunks": nch,
                                 "period_samples": int(r["period_samples"][0]),
                                 "time_bin_out": int(r["time_bin"][0])})
            arrays[f"fold{k}_intensity"] = I
            arrays[f"fold{k}_folded"] = r["folded"]
        bw, dm, f0, period, rep = SIM
        run(["simulate", bw, dm, f0, period, rep, out])
        r = O.read_records(out)
        meta["simulate"] = {"bw": bw, "dm": dm, "f0": f0, "period": period, "repeat": rep,
                            "Np": int(r["Np"][0]), "Nd": int(r["Nd"][0])}
        arrays["simulate_signal"] = r["signal"]
        arrays["simulate_signal_u16"] = r["signal_u16"]
    np.savez_compressed(os.path.join(HERE, "reference_host.npz"), **arrays)
    with open(os.path.join(HERE, "reference_host.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", os.path.join(HERE, "reference_host.npz"))


if __name__ == "__main__":
    main()
