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


class _OracleRank:
    """A rank's dedisperser with the FP64 oracle standing in for the device:
    the interface ShardedDedisperser drives (filter_block, fold_init,
    get_profiles, block_samples)."""

    def __init__(self, bw, dms, f0, fftpoint, count):
        import oracle as O
        self.O = O
        self.bw = bw
        self.d = O.Dedisp(bw, dms, f0, fftpoint, count)
        self.block_samples = self.d.count * self.d.M
        self.Nd = self.d.Nd
        self.folds = None

    def fold_init(self, period, fs, time_bin=0, discard_Nd=0, detect="power"):
        self.folds = [self.O.Fold(period, fs, self.block_samples, time_bin) for _ in range(self.d.numDMs)]
        for f in self.folds:
            f.discard_samples(int(discard_Nd))

    def filter_block(self, x):
        x = np.asarray(x)
        if x.dtype != np.complex64:
            x = self.O.decode_uint16(np.ascontiguousarray(x).view(np.uint16))
        y = self.d.filter(np.asarray(x, np.complex128))
        for f, row in zip(self.folds, y):
            f.fold_data(np.abs(row) ** 2)

    def get_profiles(self):
        return np.stack([f.fold_data_bins() for f in self.folds]).astype(np.float32)


def _sharded_worker(rank, world, port, q, kind):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from datetime import timedelta
    from msosm_gpu_b200 import shard
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        bw, f0, fftpoint, count = 16e6, 1242e6, 1024, 8
        all_dms = np.linspace(0.5, 8.0, 5).astype(np.float32)   # 3 + 2 trials over two ranks
        s = shard.ShardedDedisperser(bw, all_dms, f0, fftpoint, count, factory=lambda d: _OracleRank(
            bw, d, f0, fftpoint, count))
        s.fold_init(0.00021, bw, time_bin=16, detect="power")
        rng = np.random.default_rng(4)
        xs = []
        for c in range(8):   # past the discarded periods (max smear ~8.7k samples) into folded ones
            if kind == "c64":
                x = ((rng.standard_normal(s.block_samples) + 1j * rng.standard_normal(s.block_samples)) * 50
                     ).astype(np.complex64)
            else:
                x = np.clip(np.rint(rng.standard_normal((s.block_samples, 2)) * 500) + 32768, 1, 65535
                            ).astype(np.uint16)
            xs.append(x)
            s.filter_block(x if rank == 0 else None)   # only the source rank holds the input
        prof = s.get_profiles()
        if rank == 0:
            one = _OracleRank(bw, all_dms, f0, fftpoint, count)
            one.fold_init(0.00021, bw, time_bin=16, discard_Nd=s.max_nd())
            for x in xs:
                one.filter_block(x)
            ref = one.get_profiles()
            assert np.abs(ref).max() > 0, "nothing folded"
            q.put(("ok", prof.shape, float(np.abs(prof - ref).max() / np.abs(ref).max()), s.shard_sizes))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # pragma: no cover - surfaced through the queue
        import traceback
        q.put(("error", traceback.format_exc(), None, None))


@pytest.mark.parametrize("kind", ["c64", "u16"])
def test_sharded_dedisperser_broadcasts_input_and_gathers_profiles(kind):
    # the multi-GPU API itself over two gloo ranks: rank 0 alone holds each
    # call's input (complex64 or uint16 pairs), broadcast to rank 1; the
    # gathered profiles of the 3 + 2 trial shards equal one process over all
    # five trials
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q, kind)) for r in range(2)]
    for p in ps:
        p.start()
    try:
        status, shape, err, sizes = q.get(timeout=180)
    finally:
        for p in ps:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert status == "ok", shape
    assert tuple(shape) == (5, 16) and sizes == [2, 3]
    assert err < 1e-6
