"""Replica scheduling across processes (world size 2, gloo on CPU): every
rank derives the same partition of a batch without communicating, the
partition covers each scene once and balances pixels, and timings combine
as the maximum over ranks."""
import os
import socket

import pytest

from cuphu_b200.replicas import max_over_ranks, shard_scenes


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_scenes(sizes, rank, world)
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        t = max_over_ranks(10.0 * (rank + 1))
        q.put((rank, shards, t, sum(sizes[i] for i in mine)))
    finally:
        dist.destroy_process_group()


def test_shard_scenes_single_process():
    sizes = [512 * 512, 3072 * 3072, 1024 * 2048, 2048 * 2048, 512 * 1024]
    parts = [shard_scenes(sizes, r, 3) for r in range(3)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    assert shard_scenes(sizes, 0, 1) == list(range(len(sizes)))
    with pytest.raises(ValueError):
        shard_scenes(sizes, 3, 3)


def test_shard_and_max_over_two_gloo_ranks():
    import numpy as np
    import torch.multiprocessing as mp
    rng = np.random.default_rng(0)
    sides = (512, 1024, 2048, 3072)
    sizes = [int(rng.choice(sides)) * int(rng.choice(sides)) for _ in range(48)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    # both ranks saw the same partition, and it covers every scene once
    assert out[0][1] == out[1][1]
    flat = sorted(i for part in out[0][1] for i in part)
    assert flat == list(range(48))
    # timings combine as the max; pixel loads within one scene of each other
    assert out[0][2] == out[1][2] == 20.0
    assert abs(out[0][3] - out[1][3]) <= max(sizes)
