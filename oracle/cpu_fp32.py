"""FP32 MS-OSM / OSM coherent dedispersion on the host cores: the CPU
baseline that bench.py times beside the device paths.

TEST AND BENCHMARK INFRASTRUCTURE ONLY (like the rest of oracle/): a reported
baseline, never the product path and never its checker (the FP64 restatement
in orc.c is the checker).  It runs the reference's algorithm in single
precision -- forward FFT of overlapping windows (hop M, 2M points), per-bin
delayed product with the dedispersion filter, inverse FFT, overlap-save
discard, |y|^2 and the Fold_GPU fold -- with the reference's scaling
(product / N, unnormalised inverse, / 2M;
gpu/gpu_kernel.cu:128-198, 236-258) and its per-bin block delays and filter
(dedispersion/msosm/msosm_prepare.cpp:37-152, computed by the oracle).

FFTs: FFTW is not installed on these machines, so pocketfft (scipy.fft,
complex64 in and out) stands in for it.  Parallelism: the trials are split
over a pool of threads, one FFT worker each; numpy's array operations and
the C fold release the GIL, so all host cores work.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft as sfft

import oracle as O

FFT_LIBRARY = "pocketfft (scipy.fft %s, complex64); FFTW is not installed" % getattr(
    __import__("scipy"), "__version__", "?")


class MsosmFP32:
    """D trials of one band over one input stream, count blocks of M samples
    per call (MSOSM_GPU_DM_concurrent semantics; OSM with ``osm``), each
    trial's |y|^2 folded by the Fold_GPU state machine (float accumulation)."""

    def __init__(self, bw, dms, f0, fftpoint, count, period=None, time_bin=1024, osm=False, threads=0):
        dms = np.atleast_1d(np.asarray(dms, np.float32))
        self.D = dms.size
        self.threads = threads or os.cpu_count() or 1
        nds = [O.nd(bw, float(dm), f0) for dm in dms]
        ndmax = max(nds)
        if osm:
            M = max(O.osm_min_order(ndmax), fftpoint // 2)
        else:
            M = max(O.msosm_min_order(ndmax), fftpoint // 2)
        self.M, self.N, self.count = M, 2 * M, int(count)
        N = self.N
        # the filter carries the reference's 1/N before the unnormalised
        # inverse and its 1/2M after it; scipy's inverse divides by N itself
        self.H = np.empty((self.D, N), np.complex64)
        self.delay = np.zeros((self.D, N), np.int64)
        for i, dm in enumerate(dms):
            self.H[i] = (O.dedisp_params(bw, float(dm), f0, M) / N).astype(np.complex64)
            if not osm:
                _, dp = O.segmentation(bw, float(dm), f0, M)
                self.delay[i] = dp
        self.maxd = int(self.delay.max())
        # spectra of the last maxd + count blocks (oldest first)
        self.hist = np.zeros((self.maxd + self.count, N), np.complex64)
        self.tail = np.zeros(M, np.complex64)  # the previous call's last M samples
        # flat history index of bin b of block j for each trial: row j + maxd - delay[b]
        cols = np.arange(N)[None, :]
        self.gidx = [((np.arange(self.count)[:, None] + self.maxd - self.delay[i][None, :]) * N + cols)
                     .astype(np.int64) for i in range(self.D)]
        self.folds = None
        if period is not None:
            self.folds = [O.Fold(period, bw, self.count * M, time_bin, accumulate_float=True) for _ in range(self.D)]
            for f in self.folds:
                f.discard_samples(int(ndmax))
        self.pool = ThreadPoolExecutor(max_workers=self.threads)
        self.series = None

    def _forward(self, x):
        M, N, c = self.M, self.N, self.count
        buf = np.concatenate([self.tail, x])
        self.tail = buf[-M:].copy()
        win = np.lib.stride_tricks.as_strided(buf, shape=(c, N), strides=(M * 8, 8))
        # shift the history by count blocks and append this call's spectra
        self.hist[:-c] = self.hist[c:]

        def part(ix):
            a, b = int(ix[0]), int(ix[-1]) + 1
            self.hist[self.maxd + a:self.maxd + b] = sfft.fft(win[a:b], axis=1, workers=1)

        list(self.pool.map(part, [p for p in np.array_split(np.arange(c), min(self.threads, c)) if p.size]))

    def _trial(self, i, keep_series):
        z = np.take(self.hist.reshape(-1), self.gidx[i])
        z *= self.H[i][None, :]
        y = sfft.ifft(z, axis=1, workers=1, overwrite_x=True)[:, self.M:]
        if keep_series:
            self.series[i] = y.reshape(-1)
        if self.folds is not None:
            p = y.real * y.real + y.imag * y.imag
            self.folds[i].fold_data(np.ascontiguousarray(p.reshape(-1), np.float64))

    def filter(self, x, keep_series=False):
        """Dedisperse the next count*M complex64 samples (all trials)."""
        x = np.ascontiguousarray(x, np.complex64).reshape(-1)
        assert x.size == self.count * self.M
        self._forward(x)
        if keep_series:
            self.series = np.empty((self.D, self.count * self.M), np.complex64)
        list(self.pool.map(lambda i: self._trial(i, keep_series), range(self.D)))
        return self.series

    def profiles(self):
        return np.stack([f.fold_data_bins() for f in self.folds])

    def close(self):
        self.pool.shutdown()
