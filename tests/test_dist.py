"""Host-side multi-rank logic on CPU (gloo, world size 2): cell sharding and
the max-over-ranks timing reduction used by bench.py --gpus N."""
import os
import socket

import pytest


def test_shard_partitions_and_balances():
    from fem_b200.dist import shard
    from fem_b200 import fields
    import numpy as np
    rng = np.random.default_rng(7)
    ns = rng.choice(fields.BATCH_SIZES, size=4096, p=fields.BATCH_PROBS)
    w = [float(n) ** 3 for n in ns]
    for world in (1, 2, 4, 8):
        parts = shard(w, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(4096))
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(w)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from fem_b200.dist import max_over_ranks
        q.put((rank, max_over_ranks(10.0 + rank)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 11.0, 1: 11.0}


class _FakeEngine:
    """Engine.batch stand-in: C = mean(rho) * I, dL/drho = rho * trace(dL/dC),
    info iterations = the cell's voxel count; records the rank's cells."""

    def __init__(self):
        self.seen = []

    def batch(self, rhos, dLdC=None, allow_unconverged=False):
        import numpy as np
        self.seen.append(len(rhos))
        C = np.stack([np.eye(6) * r.mean() for r in rhos])
        infos = [{"status": 0, "iterations": [r.size] * 6} for r in rhos]
        g = None if dLdC is None else [r * np.trace(d) for r, d in zip(rhos, dLdC)]
        return C, infos, g


def _cells():
    import numpy as np
    rng = np.random.default_rng(3)
    return [rng.random((n, n, n)) for n in (4, 6, 8, 4, 6, 5, 7)]


def _batch_worker(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from fem_b200.dist import batch_sharded
        cells = _cells()
        dLdC = np.stack([np.eye(6) * (k + 1) for k in range(len(cells))])
        e = _FakeEngine()
        C, infos, g = batch_sharded(e, cells, dLdC=dLdC)
        q.put((rank, C, [i["iterations"][0] for i in infos], [x.sum() for x in g], sum(e.seen)))
    finally:
        dist.destroy_process_group()


def test_batch_sharded_gloo():
    """Two gloo ranks split 7 cells by voxels, each solves its share, and both
    end with every cell's C, info and gradient in cell order -- the same as one
    rank solving all of them."""
    import numpy as np
    import torch.multiprocessing as mp
    from fem_b200.dist import batch_sharded
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict((r[0], r[1:]) for r in (q.get(timeout=10) for _ in range(2)))
    cells = _cells()
    dLdC = np.stack([np.eye(6) * (k + 1) for k in range(len(cells))])
    C1, infos1, g1 = batch_sharded(_FakeEngine(), cells, dLdC=dLdC)   # one process, no group
    for r in (0, 1):
        C, its, gs, nseen = got[r]
        assert np.array_equal(C, C1)
        assert its == [i["iterations"][0] for i in infos1]
        assert np.allclose(gs, [x.sum() for x in g1], rtol=1e-14)
    assert got[0][3] + got[1][3] == len(cells) and min(got[0][3], got[1][3]) >= 2
