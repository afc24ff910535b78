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
