"""DM-trial sharding over ranks (one process per GPU).

Every DM trial reads the same input and is independent of the others, so the
path shards along trials: rank r dedisperses its own trials.  The input
reaches every rank once (a broadcast from one rank, or each rank's own copy)
and the folded profiles are gathered (numDMs x nbins floats); nothing else
crosses ranks.  ShardedDedisperser is that path as one object; the other
helpers are its pieces (and the max-over-ranks timing reduction).
"""
from __future__ import annotations

from typing import Tuple

import numpy as np


def world() -> Tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment."""
    import os
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def weak_trials(rank: int, n_per_rank: int, span: float, lo: float = 0.0) -> np.ndarray:
    """Weak scaling: rank r owns n_per_rank trials uniform over
    [lo + r*span, lo + (r+1)*span]."""
    return (np.linspace(lo, lo + span, n_per_rank) + rank * span).astype(np.float32)


def split_trials(dms: np.ndarray, rank: int, world_size: int) -> np.ndarray:
    """Strong scaling: contiguous shard of a fixed trial list (sizes differ by
    at most one)."""
    n = len(dms)
    lo = (n * rank) // world_size
    hi = (n * (rank + 1)) // world_size
    return np.asarray(dms[lo:hi], np.float32)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (e.g. a step time) over the process group."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_profiles(prof: np.ndarray, device=None) -> np.ndarray:
    """All ranks' profiles stacked in rank order (every rank gets the result).
    Shards must have equal shapes."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(prof, np.float32))
    if device is not None:
        t = t.to(device)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return prof
    out = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return torch.cat(out, 0).cpu().numpy()


class ShardedDedisperser:
    """One stream's DM trials over the ranks of a process group (one GPU per
    rank): rank r dedisperses its contiguous share of the trials
    (split_trials) with its own Dedisperser.  The input enters once: with
    ``broadcast`` (the default) rank ``src`` passes each call's samples and
    they are broadcast to the other ranks over the group's backend (NCCL
    between GPUs; the tensor stays on the device), otherwise every rank
    passes its own copy.  get_profiles() all-gathers the folded profiles
    into the full trial order on every rank.  Those two are the only
    collectives; nothing else crosses ranks.

    ``factory(dms) -> dedisperser`` builds a rank's dedisperser (default: a
    Dedisperser with the given arguments); anything with filter_block,
    fold_init, get_profiles and block_samples fits.
    """

    def __init__(self, bw, dms, f0, fftpoint: int = 0, count: int = 1, precision: str = "fp32",
                 series: bool = False, group=None, broadcast: bool = True, src: int = 0, device=None,
                 factory=None):
        import torch.distributed as dist
        self.group = group
        live = dist.is_available() and dist.is_initialized()
        self.world_size = dist.get_world_size(group) if live else 1
        self.rank = dist.get_rank(group) if live else 0
        self.all_dms = np.ascontiguousarray(np.atleast_1d(np.asarray(dms, np.float32)))
        if self.all_dms.size < self.world_size:
            raise ValueError(f"{self.all_dms.size} trials cannot be shared by {self.world_size} ranks")
        self.shard_sizes = [len(split_trials(self.all_dms, r, self.world_size)) for r in range(self.world_size)]
        self.dms = split_trials(self.all_dms, self.rank, self.world_size)
        self.broadcast = broadcast and self.world_size > 1
        self.src = src
        self.device = device
        self.bw, self.f0 = float(bw), float(f0)
        if factory is None:
            from .dedisp import Dedisperser

            def factory(d):
                return Dedisperser(bw, d, f0, fftpoint, count, series=series, precision=precision)
        self.d = factory(self.dms)
        self.block_samples = self.d.block_samples
        self._buf = None

    # -- the rank's own handle --------------------------------------------------
    @property
    def Nd(self) -> np.ndarray:
        return np.asarray(getattr(self.d, "Nd"))

    def max_nd(self) -> int:
        """The largest smear over ALL trials (every rank must discard the same
        periods, so folds are configured with this)."""
        from .prepare import nd
        return max(int(nd(self.bw, float(v), self.f0)) for v in self.all_dms)

    def fold_init(self, period: float, fs: float, time_bin: int = 0, discard_Nd=None, detect: str = "power"):
        self.d.fold_init(period, fs, time_bin=time_bin, discard_Nd=self.max_nd() if discard_Nd is None else discard_Nd,
                         detect=detect)

    def __getattr__(self, name):
        # set_stream, enable_timing, timing, synchronize, folded_periods, ...
        if name == "d":
            raise AttributeError(name)
        return getattr(self.d, name)

    # -- the collectives --------------------------------------------------------
    def _input_tensor(self, x):
        """This call's samples as a tensor every rank holds: complex64, or the
        offset-binary uint16 pairs as one int32 per sample.  Rank src
        broadcasts the kind, then the samples (as real numbers)."""
        import torch
        import torch.distributed as dist
        dev = self.device
        kind = torch.zeros(1, dtype=torch.int64, device=dev)
        t = None
        if self.rank == self.src:
            t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))
            if t.dtype != torch.complex64:  # uint16 pairs (or their int32 view): 4 bytes per sample
                t = t.contiguous().reshape(-1).view(torch.int32)
                kind.fill_(1)
            t = t.reshape(-1)
        dist.broadcast(kind, self.src, group=self.group)
        dtype = torch.complex64 if int(kind.item()) == 0 else torch.int32
        if self._buf is None or self._buf.dtype != dtype:
            self._buf = torch.empty(self.block_samples, dtype=dtype, device=dev)
        if t is not None:
            self._buf.copy_(t)
        dist.broadcast(torch.view_as_real(self._buf) if dtype == torch.complex64 else self._buf, self.src,
                       group=self.group)
        return self._buf

    def filter_block(self, x=None) -> None:
        """The next count*M samples: on rank ``src`` only with ``broadcast``
        (the other ranks pass None), else on every rank."""
        if self.broadcast:
            t = self._input_tensor(x)
            self.d.filter_block(t if t.is_cuda else t.numpy())
        else:
            self.d.filter_block(x)

    def get_profiles(self) -> np.ndarray:
        """[all trials, bins] on every rank (all-gather in rank order)."""
        mine = np.ascontiguousarray(self.d.get_profiles(), np.float32)
        if self.world_size == 1:
            return mine
        import torch
        import torch.distributed as dist
        width = mine.shape[1]
        m = max(self.shard_sizes)
        pad = np.zeros((m, width), np.float32)
        pad[:mine.shape[0]] = mine
        t = torch.from_numpy(pad)
        if self.device is not None:
            t = t.to(self.device)
        out = [torch.empty_like(t) for _ in range(self.world_size)]
        dist.all_gather(out, t, group=self.group)
        return np.concatenate([o.cpu().numpy()[:n] for o, n in zip(out, self.shard_sizes)], 0)

    def close(self) -> None:
        if hasattr(self.d, "close"):
            self.d.close()
