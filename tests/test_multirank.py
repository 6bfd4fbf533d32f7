"""Multi-rank host logic on CPU (gloo, world size 2): image sharding covers
every image exactly once, cost balancing, and the max-over-ranks timing."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from idi_b200.simulation.shard import max_over_ranks, shard_by_cost, shard_range


def test_shard_range_covers_all():
    for n in (0, 1, 7, 32, 33):
        for w in (1, 2, 3, 8):
            got = [shard_range(n, r, w) for r in range(w)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def test_shard_by_cost_balances_uneven_batch():
    g = np.random.Generator(np.random.Philox(1))
    counts = np.floor(np.exp(g.uniform(np.log(1e3), np.log(1e5), 256))).astype(int)
    parts = shard_by_cost(counts, 8)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(256))
    loads = [counts[p].sum() for p in parts]
    assert max(loads) / np.mean(loads) < 1.02
    assert shard_by_cost(counts, 8) == parts  # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        start, stop = shard_range(32, rank, world)
        # every rank times its own shard; the job time is the slowest rank
        t = max_over_ranks(1.5 + rank)
        q.put((rank, start, stop, t))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_sharding_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res[0][1:3] == (0, 16) and res[1][1:3] == (16, 32)
    assert res[0][3] == res[1][3] == 2.5
    assert max_over_ranks(3.0) == 3.0  # no process group in the parent
