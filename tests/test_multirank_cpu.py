"""The multi-rank path on CPU: two gloo ranks shard DM trials, dedisperse
their shard (with the oracle standing in for the device, which this test does
not need), reduce the step time with MAX and gather the folded profiles; rank
0 checks the union equals one process over all trials."""
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from datetime import timedelta
    import oracle as O
    from msosm_gpu_b200 import shard
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        ws, r, _ = shard.world()
        assert (ws, r) == (world, rank)
        all_dms = np.linspace(0.5, 8.0, 6).astype(np.float32)
        mine = shard.split_trials(all_dms, rank, world)
        x = (np.random.default_rng(3).standard_normal(8192) * 50).astype(np.complex128)
        d = O.Dedisp(16e6, mine, 1242e6, 1024, 8)
        prof = []
        for c in range(2):
            y = d.filter(x[c * 4096:(c + 1) * 4096])
            prof.append((np.abs(y) ** 2).reshape(len(mine), -1, 64).sum(1))
        prof = np.sum(prof, 0).astype(np.float32)
        t = shard.max_over_ranks(1.0 + rank)
        allp = shard.gather_profiles(prof)
        if rank == 0:
            full = O.Dedisp(16e6, all_dms, 1242e6, 1024, 8)
            ref = []
            for c in range(2):
                y = full.filter(x[c * 4096:(c + 1) * 4096])
                ref.append((np.abs(y) ** 2).reshape(len(all_dms), -1, 64).sum(1))
            ref = np.sum(ref, 0).astype(np.float32)
            q.put(("ok", t, float(np.abs(allp - ref).max() / np.abs(ref).max()),
                   shard.weak_trials(1, 4, 100.0).tolist()))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # pragma: no cover - surfaced through the queue
        q.put(("error", repr(e), None, None))


def test_two_gloo_ranks_shard_dm_trials():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    try:
        status, t, err, weak = q.get(timeout=180)
    finally:
        for p in ps:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert status == "ok", t
    assert t == 2.0
    assert err < 1e-6
    assert weak == pytest.approx([100.0, 133.33333, 166.66667, 200.0], rel=1e-5)
