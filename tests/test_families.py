"""Host logic of the batching form: the family generator and the sharding of
whole systems over ranks (no data-path collective: each rank solves its own
systems), checked with two gloo ranks on the CPU."""
import os

import numpy as np
import pytest

import families


def test_shard_covers_every_system_once():
    w = [float(v) for v in np.random.default_rng(0).integers(1, 1000, 64)]
    for world in (1, 2, 3, 8):
        parts = families.shard(w, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) <= sum(w) / world + max(w)


def test_batch_member_shapes():
    A, nv, B = families.batch_member(7, 6, 12)
    n = A.nrows
    side = round(n ** (1 / 3))
    assert side ** 3 == n and 6 <= side <= 12
    assert nv in (1, 2, 4, 8) and B.shape == (n, nv)
    rp, ci, v = A.arrays()
    assert np.all(ci[rp[:-1]] == np.arange(n))  # diagonal first
    assert np.all(v[rp[:-1]] > 0)


def _rank(rank, world, port, weights, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = families.shard(weights, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    dist.destroy_process_group()
    q.put((rank, got))


def test_two_gloo_ranks_agree_on_disjoint_shards():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    w = [float(v) for v in np.random.default_rng(1).integers(1, 500, 64)]
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, w, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert res[0] == res[1]
    a, b = res[0]
    assert set(a).isdisjoint(b) and sorted(a + b) == list(range(64))
