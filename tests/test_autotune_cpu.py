"""Host logic of the autotuner and of the uneven-batch workload (no GPU):
candidate sets follow the MS-OSM minimum order and the error budget; fixed
configurations are raised to an observation's minimum and fall back to FP32
where the tensor path has no kernel; the workload's observations follow
their stated distributions."""
import numpy as np
import pytest

import bench
from msosm_gpu_b200 import autotune as A
from msosm_gpu_b200.prepare import msosm_min_order, nd


def test_candidates_respect_minimum_and_budget():
    dms = np.linspace(0, 100, 64).astype(np.float32)
    m_min = max(msosm_min_order(nd(16e6, float(d), 1242e6)) for d in dms)
    c = A.candidates(16e6, dms, 1242e6)
    assert all(n >= 2 * m_min for n, _ in c)
    assert (4096, "fp16") in c and (8192, "fp16") in c
    assert not any(p == "bf16" for _, p in c)  # bf16 profiles exceed 1e-3
    assert any(p == "bf16" for _, p in A.candidates(16e6, dms, 1242e6, budget=5e-3))
    assert [p for _, p in A.candidates(16e6, dms, 1242e6, budget=1e-5)] == ["fp32"] * len(
        {n for n, _ in c})
    # a long smear leaves the tensor cores only their largest size, 16384
    big = A.candidates(64e6, [300.0], 1068e6)
    assert all(n >= 16384 for n, _ in big) and any(n > 16384 for n, _ in big)
    assert {n for n, p in big if p != "fp32"} == {16384}


def test_fixed_choice():
    assert A.fixed_choice(16e6, [50.0], 1242e6, 4096, "fp16") == (4096, "fp16")
    assert A.fixed_choice(64e6, [300.0], 1068e6, 4096, "fp16") == (16384, "fp16")
    # above the tensor path's sizes the fixed choice falls back to FP32
    assert A.fixed_choice(64e6, [300.0], 1068e6, 32768, "fp16") == (32768, "fp32")
    assert A.fixed_choice(16e6, [1.0], 1242e6, 2048, "fp32") == (2048, "fp32")


def test_uneven_observations():
    obs = bench.uneven_observations(64, 0)
    assert len(obs) == 64
    n = np.array([o["n"] for o in obs])
    assert n.min() >= 1 << 19 and n.max() <= 1 << 25 and np.all(n % (1 << 15) == 0)
    assert {o["bw"] for o in obs} <= {4e6, 16e6, 32e6, 64e6}
    for o in obs:
        assert 1100e6 <= o["f0"] + o["bw"] / 2 <= 1500e6 + 1
        assert 16 <= o["trials"] <= 512 and 20 <= o["dm_max"] <= 300
        assert 0 < o["dm"] <= 0.9 * o["dm_max"] and 1e-3 <= o["period"] <= 1.0
    assert obs == bench.uneven_observations(64, 0)


def test_coherence_floor_drops_the_coarsest_sizes():
    from msosm_gpu_b200.autotune import candidates, coherence
    bw, f0 = 16e6, 1242e6
    dms = np.linspace(0.0, 100.0, 16)
    all_sizes = sorted({n for n, _ in candidates(bw, dms, f0)})
    assert all_sizes[0] == 2048
    # FFT 2048 keeps ~0.92 of the exact filter's coherence at DM 100, 4096 ~0.96
    assert 0.90 < coherence(bw, 100.0, f0, 2048) < 0.94 < coherence(bw, 100.0, f0, 4096) < 0.98
    kept = sorted({n for n, _ in candidates(bw, dms, f0, min_coherence=0.95)})
    assert kept == [n for n in all_sizes if n >= 4096]
    with pytest.raises(ValueError):
        candidates(bw, dms, f0, sizes=(2048,), min_coherence=0.95)
