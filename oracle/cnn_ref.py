"""CPU restatement of the DM-proposal network (numpy, FP64).

TEST INFRASTRUCTURE ONLY: the checker of the device network
(msosm_gpu_b200/csrc/cnn.cu).  Only tests/ import it.

Network: input x [B, Cin, L] (folded profiles of Cin coarse DM trials, L
phase bins); `layers` circular 'same' 1-D convolutions of `channels` outputs
and kernel K, each followed by ReLU; the mean over phase; two linear heads:
a detection logit and a DM offset.  Loss: mean over the batch of the
logistic loss of the logit against the label, plus `dm_weight` times the
mean over positive samples of the squared offset error.

Parameters, one flat float32 vector in this order: for each layer the
weights [C_out][C_in][K] and biases [C_out]; then the detection head
weights [C] and bias [1]; then the offset head weights [C] and bias [1].
Weights are used rounded to bf16 (round to nearest even); biases as they
are.
"""
from __future__ import annotations

import numpy as np


def shapes(cin: int, channels: int, kernel: int, layers: int):
    out = []
    ci = cin
    for _ in range(layers):
        out.append(("w", (channels, ci, kernel)))
        out.append(("b", (channels,)))
        ci = channels
    out += [("w", (channels,)), ("b", (1,)), ("w", (channels,)), ("b", (1,))]
    return out


def unpack(theta: np.ndarray, cin, channels, kernel, layers, quantise=True):
    ps, o = [], 0
    for kind, shp in shapes(cin, channels, kernel, layers):
        n = int(np.prod(shp))
        v = np.asarray(theta[o:o + n], np.float32 if quantise else np.float64).reshape(shp)
        if kind == "w" and quantise:
            v = bf16(v)
        ps.append(v.astype(np.float64))
        o += n
    return ps


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> bf16 (round to nearest even) -> float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _cols(x, K):
    B, C, L = x.shape
    p = K // 2
    xp = np.concatenate([x[:, :, L - p:], x, x[:, :, :p]], axis=2)
    return np.stack([xp[:, :, k:k + L] for k in range(K)], axis=3)  # [B, C, L, K]


def forward(theta, x, cin, channels, kernel, layers, quantise=True):
    ps = unpack(theta, cin, channels, kernel, layers, quantise)
    a = np.asarray(x, np.float64)
    acts = [a]
    for l in range(layers):
        w, b = ps[2 * l], ps[2 * l + 1]
        z = np.einsum("bclk,ock->bol", _cols(a, kernel), w) + b[None, :, None]
        a = np.maximum(z, 0.0)
        acts.append(a)
    h = a.mean(axis=2)
    wd, bd, wr, br = ps[2 * layers:]
    return h @ wd + bd[0], h @ wr + br[0], acts, h, ps


def loss_and_grad(theta, x, label, target, cin, channels, kernel, layers, dm_weight, quantise=True):
    logit, off, acts, h, ps = forward(theta, x, cin, channels, kernel, layers, quantise)
    B = x.shape[0]
    label = np.asarray(label, np.float64)
    pos = label > 0.5
    npos = max(1, int(pos.sum()))
    # logistic loss, numerically stable
    lo = np.maximum(logit, 0) - logit * label + np.log1p(np.exp(-np.abs(logit)))
    err = off - np.asarray(target, np.float64)
    loss = lo.mean() + dm_weight * np.sum(np.where(pos, err * err, 0.0)) / npos
    dlogit = (1.0 / (1.0 + np.exp(-logit)) - label) / B
    doff = dm_weight * 2.0 * np.where(pos, err, 0.0) / npos
    wd, bd, wr, br = ps[2 * layers:]
    grads = [None] * len(ps)
    grads[2 * layers] = h.T @ dlogit
    grads[2 * layers + 1] = np.array([dlogit.sum()])
    grads[2 * layers + 2] = h.T @ doff
    grads[2 * layers + 3] = np.array([doff.sum()])
    dh = np.outer(dlogit, wd) + np.outer(doff, wr)  # [B, C]
    L = x.shape[2]
    g = np.repeat(dh[:, :, None], L, axis=2) / L * (acts[layers] > 0)  # d pre-activation of the last layer
    p = kernel // 2
    for l in range(layers - 1, -1, -1):
        a = acts[l]
        w = ps[2 * l]
        grads[2 * l] = np.einsum("bol,bclk->ock", g, _cols(a, kernel))
        grads[2 * l + 1] = g.sum(axis=(0, 2))
        if l > 0:
            # dx[b, c, s] = sum_o sum_k w[o, c, k] g[b, o, s - k + p]
            gp = np.concatenate([g[:, :, L - p:], g, g[:, :, :p]], axis=2)
            dx = np.zeros_like(a)
            for k in range(kernel):
                # s - k + p = t -> g index t + p in gp shifted: gp[:, :, s - k + 2p]
                sh = gp[:, :, 2 * p - k: 2 * p - k + L]
                dx += np.einsum("oc,bol->bcl", w[:, :, k], sh)
            g = dx * (a > 0)
    flat = np.concatenate([gr.reshape(-1) for gr in grads])
    return loss, flat, logit, off
