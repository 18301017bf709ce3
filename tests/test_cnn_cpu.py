"""Host side of the DM-proposal network: the numpy restatement's gradients
against finite differences, its bf16 rounding, and the C ABI's argument
checks (no GPU needed)."""
import ctypes

import numpy as np
import pytest

import cnn_ref as R
from msosm_gpu_b200 import _abi
from msosm_gpu_b200._abi import lib
from msosm_gpu_b200.dm_proposal import normalise, profile_snr


def test_restatement_gradient_by_finite_differences():
    rng = np.random.default_rng(0)
    cin, ch, K, lay, L, B = 5, 4, 7, 3, 16, 6
    n = sum(int(np.prod(s)) for _, s in R.shapes(cin, ch, K, lay))
    th = rng.standard_normal(n) * 0.3
    x = rng.standard_normal((B, cin, L))
    y = (rng.random(B) > 0.5).astype(float)
    t = rng.standard_normal(B)
    _, g, _, _ = R.loss_and_grad(th, x, y, t, cin, ch, K, lay, 0.7, quantise=False)
    eps = 1e-6
    for i in rng.choice(n, 60, replace=False):
        tp, tm = th.copy(), th.copy()
        tp[i] += eps
        tm[i] -= eps
        fd = (R.loss_and_grad(tp, x, y, t, cin, ch, K, lay, 0.7, quantise=False)[0]
              - R.loss_and_grad(tm, x, y, t, cin, ch, K, lay, 0.7, quantise=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd))


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30], np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # ties to even
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert abs(r[3] + 3.14159) < 2 ** -7 * 4


@pytest.mark.parametrize("field,value", [("in_channels", 12), ("length", 40), ("channels", 4), ("kernel", 6),
                                         ("layers", 0), ("max_batch", 2048)])
def test_config_rejected(field, value):
    cfg = _abi.CnnConfig(64, 256, 32, 7, 4, 256, 0.25)
    setattr(cfg, field, value)
    h = ctypes.c_void_p()
    assert lib().msosm_cnn_create(ctypes.byref(cfg), 0, ctypes.byref(h)) == _abi.ERR_BAD_ARG


def test_host_helpers():
    rng = np.random.default_rng(1)
    p = rng.standard_normal((8, 256)) + 5
    x = normalise(p)
    assert np.allclose(x.mean(axis=1), 0, atol=1e-6) and abs(x.std() - 1) < 1e-5
    q = rng.standard_normal(256)
    q[100:110] += 4
    assert profile_snr(q, 10) > 8
