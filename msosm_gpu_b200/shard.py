"""DM-trial sharding over ranks (one process per GPU).

Every DM trial reads the same input and is independent of the others, so the
path shards along trials with no data-path exchange: rank r dedisperses its
own trials over its own copy of the input.  The only collectives are the
max-over-ranks timing reduction and, for users who want all profiles on one
rank, a gather of the folded profiles (numDMs x nbins floats per rank).
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
