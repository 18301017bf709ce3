"""The tensor-core row order on the host: tc_pos (csrc/tc_layout.hpp) is a
permutation at FFT 4096, 8192 and 16384, and every bin pair a gather thread
reads is the one whose GEMM operand element it writes (tests/cpp/
tc_layout_check.cpp, compiled with g++ against the kernel's own header)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tc_row_order_matches_gather(tmp_path):
    exe = str(tmp_path / "tc_layout_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "msosm_gpu_b200", "csrc"),
                    "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "tc_layout_check.cpp"),
                    "-o", exe], check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
