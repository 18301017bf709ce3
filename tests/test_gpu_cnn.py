"""The DM-proposal network's kernels against their numpy restatement
(oracle/cnn_ref.py, FP64 with the same bf16-rounded weights): forward
values, every parameter's gradient, one Adam step; run-to-run bit identity;
and that the network learns a separable toy problem."""
import numpy as np
import pytest

import cnn_ref as R
from msosm_gpu_b200.dm_proposal import DMProposalNet

pytestmark = pytest.mark.gpu

SHAPE = dict(in_channels=16, length=64, channels=16, kernel=7, layers=3)


def batch(rng, B, cin, L):
    x = rng.standard_normal((B, cin, L)).astype(np.float32)
    y = (rng.random(B) > 0.5).astype(np.float32)
    t = rng.standard_normal(B).astype(np.float32)
    return x, y, t


@pytest.mark.parametrize("B", [1, 8, 40])
def test_forward_and_gradient_match_oracle(B):
    net = DMProposalNet(**SHAPE, max_batch=64, dm_weight=0.5, seed=3)
    rng = np.random.default_rng(B)
    th = net.params()
    # non-zero biases so every parameter is exercised
    th = th + rng.standard_normal(th.size).astype(np.float32) * 0.05
    net.set_params(th)
    x, y, t = batch(rng, B, SHAPE["in_channels"], SHAPE["length"])
    logit, off = net.forward(x)
    a = (SHAPE["in_channels"], SHAPE["channels"], SHAPE["kernel"], SHAPE["layers"])
    rl, ro, _, _, _ = R.forward(th, x, *a)
    np.testing.assert_allclose(logit, rl, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(off, ro, rtol=1e-4, atol=1e-5)
    loss, g = net.gradient(x, y, t, want_grad=True)
    rloss, rg, _, _ = R.loss_and_grad(th, x, y, t, *a, 0.5)
    assert abs(loss - rloss) <= 1e-5 * max(1.0, abs(rloss))
    # per parameter block: relative error of the block's gradient
    o = 0
    for kind, shp in R.shapes(*a):
        n = int(np.prod(shp))
        gb, rb = g[o:o + n].astype(np.float64), rg[o:o + n]
        err = np.linalg.norm(gb - rb) / max(np.linalg.norm(rb), 1e-12)
        assert err < 1e-4, (kind, shp, err)
        o += n
    net.close()


def test_adam_step_and_determinism():
    net = DMProposalNet(**SHAPE, max_batch=32, dm_weight=0.5, seed=5)
    rng = np.random.default_rng(9)
    x, y, t = batch(rng, 32, SHAPE["in_channels"], SHAPE["length"])
    th0 = net.params()
    l1, g1 = net.gradient(x, y, t, want_grad=True)
    l2, g2 = net.gradient(x, y, t, want_grad=True)
    assert l1 == l2 and np.array_equal(g1, g2)
    net.step(x, y, t, 1e-3)
    th1 = net.params()
    # Adam's first step: m = 0.1 g, v = 0.001 g^2, bias-corrected -> g / (|g| + eps')
    want = th0 - 1e-3 * g1 / (np.sqrt(g1.astype(np.float64) ** 2) + 1e-8)
    np.testing.assert_allclose(th1, want, rtol=1e-5, atol=1e-7)
    net.close()


def test_learns_a_toy_problem():
    """Positives carry a pulse in one input channel at a random phase, with
    the target the channel index; the network must separate them."""
    rng = np.random.default_rng(0)
    cin, L, n = 16, 64, 1024
    X = rng.standard_normal((n, cin, L)).astype(np.float32) * 0.5
    y = (rng.random(n) > 0.5).astype(np.float32)
    t = np.zeros(n, np.float32)
    for i in np.nonzero(y)[0]:
        c, ph = rng.integers(cin), rng.integers(L)
        X[i, c, (ph + np.arange(4)) % L] += 3.0
        t[i] = c / cin
    net = DMProposalNet(cin, L, 16, 7, 3, max_batch=128, dm_weight=1.0, seed=1)
    for ep in range(25):
        perm = rng.permutation(n)
        for s in range(0, n, 128):
            idx = perm[s:s + 128]
            net.step(np.ascontiguousarray(X[idx]), y[idx], t[idx], 3e-3)
    lg, of = net.forward(np.ascontiguousarray(X[:128]))
    acc = np.mean((lg > 0) == (y[:128] > 0.5))
    assert acc > 0.95, acc
    net.close()


def test_network_gain_over_coarse_peak_search():
    """Trained on simulated observations (half noise only) at a small scale,
    the network's detection head lets the search skip most noise-only
    observations: fewer fine trials per observation than searching around
    every coarse peak, at about the same recall of the pulsars the
    exhaustive fine sweep detects."""
    import torch
    from msosm_gpu_b200 import dm_proposal as P
    from msosm_gpu_b200.simulator import pulsar_baseband
    band = P.Band(bw=16e6, f0=1242e6, samples=1 << 22, dm_max=100.0, coarse=32, nbins=128, fftpoint=4096)
    ranges = dict(period=(2e-3, 30e-3), duty=(0.02, 0.08), snr=(0.03, 0.3))
    X, lab, tgt, _ = P.simulate_profiles(512, band, seed=11, **ranges)
    net = P.DMProposalNet(band.coarse, band.nbins, 32, 7, 4, max_batch=128, dm_weight=0.25, seed=2)
    P.train(net, X, lab, tgt, epochs=30, batch=128, lr=2e-3)
    rng = np.random.default_rng(12)
    cs = band.dm_max / (band.coarse - 1)
    fine = band.dm_max / 1023
    rows = []
    for i in range(40):
        p = P.draw_pulsar(rng, band, **ranges)
        pulsar = i % 2 == 0
        x = pulsar_baseband(band.samples, band.bw, band.f0, p["dm"], p["period"], p["duty"],
                            p["snr"] if pulsar else 0.0, seed=5000 + i, device=torch.device("cuda"))
        prof = P.fold_trials(x, band, band.coarse_dms, p["period"])
        lg, of = net.forward(np.ascontiguousarray(P.normalise(prof)[None]))
        k = P.coarse_peak(prof, p["duty"])
        r = dict(pulsar=pulsar, flag=bool(lg[0] > 0))
        if pulsar:
            _, snr = P.fine_search(x, band, p["period"], p["duty"], 0.0, band.dm_max, fine)
            r["sweep"] = float(snr.max())
            for name, c in (("base", k * cs), ("net", (k + float(of[0])) * cs)):
                _, ws = P.fine_search(x, band, p["period"], p["duty"], c - 2 * cs, c + 2 * cs, fine)
                r[name] = bool(ws.size and ws.max() >= 0.9 * r["sweep"])
        rows.append(r)
        del x
    det = [r for r in rows if r["pulsar"] and r["sweep"] >= 8]
    noise = [r for r in rows if not r["pulsar"]]
    assert len(det) >= 12, len(det)
    base_recall = np.mean([r["base"] for r in det])
    net_recall = np.mean([r["net"] and r["flag"] for r in det])
    noise_skipped = np.mean([not r["flag"] for r in noise])
    win = int(4 * cs / fine) + 1
    base_trials = band.coarse + win
    net_trials = band.coarse + win * np.mean([r["flag"] for r in rows])
    print(f"recall base {base_recall:.2f} net {net_recall:.2f}; noise skipped {noise_skipped:.2f}; "
          f"trials per observation base {base_trials} net {net_trials:.1f}")
    assert noise_skipped >= 0.8
    assert net_trials < 0.75 * base_trials
    assert net_recall >= base_recall - 0.15
    net.close()
