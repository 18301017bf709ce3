"""Learned DM proposal: a small 1-D CNN reads the folded profiles of a
coarse DM grid and proposes where to run fine coherent trials.

* ``DMProposalNet``: the network of ``msosm_cnn_*`` (4 circular convolutions
  of 32 channels, kernel 7, ReLU, mean over phase, a detection head and a
  DM-offset head; bf16 weights, FP32 accumulation), trained by its own
  forward and backward kernels with Adam.
* ``simulate_profiles``: pulsars (and noise-only samples) from the device
  simulator, dedispersed at the coarse trials and folded at the pulsar's
  period by the batched MS-OSM path; the network's input is the normalised
  [coarse trials x phase bins] profile stack, its targets the label and the
  offset of the true DM from the coarse trial of highest boxcar S/N, in
  coarse steps, clipped to +-OFFSET_CLIP.
* ``fine_search``: MS-OSM trials on a fine grid over a DM window, with the
  S/N of each trial's profile; the exhaustive search is the same over the
  whole range and judges the proposal's recall and DM error.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import check, lib

OFFSET_CLIP = 3.0  # coarse steps


def _ptr(a):
    if a is None:
        return None
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


class DMProposalNet:
    def __init__(self, in_channels: int = 64, length: int = 256, channels: int = 32, kernel: int = 7,
                 layers: int = 4, max_batch: int = 256, dm_weight: float = 0.25, seed: int = 0):
        self.cfg = _abi.CnnConfig(in_channels, length, channels, kernel, layers, max_batch, dm_weight)
        h = ctypes.c_void_p()
        check(lib().msosm_cnn_create(ctypes.byref(self.cfg), seed, ctypes.byref(h)))
        self._h = h
        n = ctypes.c_size_t()
        check(lib().msosm_cnn_param_count(self._h, ctypes.byref(n)))
        self.n_params = int(n.value)

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        check(lib().msosm_cnn_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        check(lib().msosm_cnn_set_params(self._h, p.ctypes.data))

    def forward(self, x):
        """x: [B, in_channels, length] float32 (host array or device tensor)."""
        B = x.shape[0]
        logit = np.empty(B, np.float32)
        off = np.empty(B, np.float32)
        check(lib().msosm_cnn_forward(self._h, _ptr(x), B, logit.ctypes.data, off.ctypes.data))
        return logit, off

    def gradient(self, x, label, target, want_grad: bool = False):
        B = x.shape[0]
        loss = ctypes.c_float()
        g = np.empty(self.n_params, np.float32) if want_grad else None
        check(lib().msosm_cnn_gradient(self._h, _ptr(x), _ptr(label), _ptr(target), B, ctypes.byref(loss),
                                       None if g is None else g.ctypes.data))
        return float(loss.value), g

    def step(self, x, label, target, lr: float) -> float:
        loss, _ = self.gradient(x, label, target)
        check(lib().msosm_cnn_adam_step(self._h, float(lr)))
        return loss

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().msosm_cnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# data: coarse-DM folded profiles of simulated observations
# ---------------------------------------------------------------------------

@dataclass
class Band:
    bw: float = 32e6
    f0: float = 1384e6           # lower edge: centre 1400 MHz
    samples: int = 1 << 24
    dm_max: float = 500.0
    coarse: int = 64
    nbins: int = 256
    fftpoint: int = 8192
    precision: str = "fp16"

    @property
    def coarse_dms(self) -> np.ndarray:
        return np.linspace(0.0, self.dm_max, self.coarse).astype(np.float32)


def profile_snr(p: np.ndarray, width: int) -> float:
    """Boxcar S/N of one folded profile (circular, off-pulse from the bins
    more than two widths away)."""
    p = np.asarray(p, np.float64)
    n = p.size
    c = np.concatenate([p, p[:width - 1]])
    box = np.convolve(c, np.ones(width), "valid")[:n]
    k = int(np.argmax(box))
    mask = np.ones(n, bool)
    mask[(np.arange(-2 * width, 3 * width) + k) % n] = False
    off = p[mask]
    sd = off.std()
    return float((box[k] - width * off.mean()) / (sd * math.sqrt(width))) if sd > 0 else 0.0


def normalise(prof: np.ndarray) -> np.ndarray:
    """[trials, bins] -> zero mean per trial, unit deviation over the stack."""
    x = prof.astype(np.float64)
    x -= x.mean(axis=1, keepdims=True)
    s = x.std()
    return (x / s if s > 0 else x).astype(np.float32)


_HANDLES: "dict" = {}   # trial grid -> Dedisperser, most recently used last
_HANDLE_CACHE = 9  # the coarse grid, the sweep's chunks and the windows of one observation


def _handle(band: Band, dms: np.ndarray):
    """A dedisperser for this band and trial grid, reset for a new stream:
    kept across observations (the filters and ring of a grid are designed
    and allocated once), at most _HANDLE_CACHE grids."""
    from .dedisp import Dedisperser
    key = (band.bw, band.f0, band.fftpoint, band.samples, band.precision, dms.tobytes())
    d = _HANDLES.pop(key, None)
    if d is None:
        while len(_HANDLES) >= _HANDLE_CACHE:
            _HANDLES.pop(next(iter(_HANDLES))).close()
        d = Dedisperser(band.bw, dms, band.f0, band.fftpoint, count=band.samples // (band.fftpoint // 2),
                        series=False, precision=band.precision)
    else:
        d.reset()
    _HANDLES[key] = d
    return d


def release_handles() -> None:
    """Free the dedispersers kept by fold_trials."""
    while _HANDLES:
        _HANDLES.pop(next(iter(_HANDLES))).close()


def fold_trials(x, band: Band, dms: Sequence[float], period: float, nbins: Optional[int] = None) -> np.ndarray:
    """Folded |y|^2 profiles [len(dms), nbins] of one observation (device
    tensor of band.samples complex64) at the given trials."""
    M = band.fftpoint // 2
    nb = nbins or band.nbins
    ps = int(np.float32(period) * np.float32(band.bw))
    nb = min(nb, ps)
    d = _handle(band, np.ascontiguousarray(np.asarray(dms, np.float32)))
    info = d.info()
    d.fold_init(period, band.bw, time_bin=nb, discard_Nd=int(info.max_delaycount) * M, detect="power")
    d.filter_block(x)
    return d.get_profiles()


def draw_pulsar(rng, band: Band, dm_range=None, period=(1e-3, 1.0), duty=(0.01, 0.10), snr=(0.01, 0.2)):
    lo, hi = dm_range or (0.0, band.dm_max)
    return dict(dm=float(rng.uniform(lo, hi)),
                period=float(math.exp(rng.uniform(math.log(period[0]), math.log(period[1])))),
                duty=float(rng.uniform(*duty)), snr=float(rng.uniform(*snr)))


def coarse_peak(prof: np.ndarray, duty: float) -> int:
    """The coarse trial of highest boxcar S/N (width = duty x bins)."""
    w = max(1, int(round(duty * prof.shape[1])))
    return int(np.argmax([profile_snr(q, w) for q in prof]))


def simulate_profiles(n: int, band: Band, seed: int = 0, noise_fraction: float = 0.5, **ranges):
    """n samples: (X [n, coarse, nbins] float32, label [n], target [n], meta).
    Noise-only samples fold pure noise at a random period."""
    import torch
    from .simulator import pulsar_baseband
    rng = np.random.default_rng(seed)
    X = np.zeros((n, band.coarse, band.nbins), np.float32)
    label = np.zeros(n, np.float32)
    target = np.zeros(n, np.float32)
    meta = []
    step = band.dm_max / (band.coarse - 1)
    dev = torch.device("cuda")
    import sys
    import time
    t0 = time.time()
    for i in range(n):
        if i and i % 2000 == 0:
            print(f"simulate_profiles: {i}/{n} in {time.time() - t0:.0f} s", file=sys.stderr, flush=True)
        p = draw_pulsar(rng, band, **ranges)
        pulsar = rng.random() >= noise_fraction
        x = pulsar_baseband(band.samples, band.bw, band.f0, p["dm"], p["period"], p["duty"],
                            p["snr"] if pulsar else 0.0, seed=int(rng.integers(1 << 62)), device=dev)
        prof = fold_trials(x, band, band.coarse_dms, p["period"])
        if prof.shape[1] < band.nbins:  # a period shorter than nbins samples
            prof = np.repeat(prof, -(-band.nbins // prof.shape[1]), axis=1)[:, :band.nbins]
        X[i] = normalise(prof)
        label[i] = 1.0 if pulsar else 0.0
        k = coarse_peak(prof, p["duty"])
        target[i] = float(np.clip((p["dm"] - k * step) / step, -OFFSET_CLIP, OFFSET_CLIP)) if pulsar else 0.0
        meta.append(dict(p, pulsar=bool(pulsar), peak_trial=k))
        del x
    return X, label, target, meta


def train(net: DMProposalNet, X, label, target, epochs: int = 30, batch: int = 256, lr: float = 2e-3, seed: int = 0,
          log=None):
    """Adam over shuffled minibatches; returns the mean loss per epoch."""
    import torch
    rng = np.random.default_rng(seed)
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    Ld = torch.from_numpy(np.ascontiguousarray(label)).cuda()
    Td = torch.from_numpy(np.ascontiguousarray(target)).cuda()
    n = X.shape[0]
    hist = []
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).cuda()
        tot, nb = 0.0, 0
        for s in range(0, n - batch + 1, batch):
            idx = perm[s:s + batch]
            xb, lb, tb = Xd[idx].contiguous(), Ld[idx].contiguous(), Td[idx].contiguous()
            torch.cuda.synchronize()
            tot += net.step(xb, lb, tb, lr)
            nb += 1
        hist.append(tot / max(nb, 1))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.4f}")
    return hist


def predict(net: DMProposalNet, X, batch: int = 256):
    logits, offs = [], []
    for s in range(0, X.shape[0], batch):
        lg, of = net.forward(np.ascontiguousarray(X[s:s + batch]))
        logits.append(lg)
        offs.append(of)
    return np.concatenate(logits), np.concatenate(offs)


def fine_search(x, band: Band, period: float, duty: float, lo: float, hi: float, step: float,
                chunk: int = 1024):
    """(trials, S/N per trial) of fine MS-OSM trials over [lo, hi]."""
    dms = np.arange(max(lo, 0.0), min(hi, band.dm_max) + 1e-9, step, dtype=np.float64).astype(np.float32)
    w = max(1, int(round(duty * band.nbins)))
    snr = np.zeros(dms.size)
    for s in range(0, dms.size, chunk):
        prof = fold_trials(x, band, dms[s:s + chunk], period)
        ww = max(1, int(round(duty * prof.shape[1])))
        snr[s:s + chunk] = [profile_snr(p, ww) for p in prof]
    return dms, snr
