"""How closely MS-OSM follows exact coherent dedispersion, with the FP64
oracle: the reference's method (MS-OSM at FFT 2M, msosm_prepare.cpp) against
classical overlap-save with the full-length filter (N = 2 nextpow2(Nd),
osm_prepare.cpp) on the same noise, past the first Nd samples.  The outputs
are aligned (cross-correlation peak at lag 0), and their coherence
rho = |<a, b>| / (|a| |b|) follows 1 - rho ~ 0.24 sqrt(Nd) / M: the
multi-segment approximation's error falls as 1/M.  This is what the
autotuner's coherence floor models (msosm_gpu_b200/autotune.py)."""
import math

import numpy as np
import pytest

import oracle as O
from msosm_gpu_b200.autotune import COHERENCE_SLOPE, coherence


def coherences(bw, dm, f0, doublings):
    Nd = O.nd(bw, dm, f0)
    m_min = O.msosm_min_order(Nd)
    osm_m = O.osm_min_order(Nd)
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(2 * osm_m) + 1j * rng.standard_normal(2 * osm_m)) * 100
    d = O.Dedisp(bw, [dm], f0, 2 * osm_m, count=1, osm=True)
    ref = np.concatenate([d.filter(x[c * osm_m:(c + 1) * osm_m])[0] for c in range(2)])
    s = slice(Nd + 4096, 2 * osm_m)
    out = []
    for k in range(doublings):
        M = m_min << k
        d = O.Dedisp(bw, [dm], f0, 2 * M, count=osm_m // M)
        y = np.concatenate([d.filter(x[c * osm_m:(c + 1) * osm_m])[0] for c in range(2)])
        a, b = y[s], ref[s]
        out.append((M, float(np.abs(np.vdot(a, b)) / (np.linalg.norm(a) * np.linalg.norm(b)))))
    return Nd, out


@pytest.mark.parametrize("bw,dm,f0,doublings", [(16e6, 100.0, 1242e6, 5), (64e6, 80.0, 1368e6, 3)])
def test_msosm_coherence_with_exact_dedispersion(bw, dm, f0, doublings):
    Nd, rows = coherences(bw, dm, f0, doublings)
    rhos = [r for _, r in rows]
    assert all(b > a for a, b in zip(rhos, rhos[1:]))  # larger M, closer to exact
    for M, rho in rows:
        model = COHERENCE_SLOPE * math.sqrt(Nd) / M
        assert abs((1 - rho) - model) < 0.25 * model, (M, rho, model)
        assert abs(coherence(bw, dm, f0, 2 * M) - (1 - model)) < 1e-12
