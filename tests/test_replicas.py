"""Replica plumbing on CPU: the case partition and the max-over-ranks timing
reduction with two gloo ranks (no GPU)."""

import os
import socket

import pytest

from up3d_b200.replicas import max_over_ranks, shard


def test_shard_partitions_every_item_once():
    for n in (0, 1, 5, 48, 49):
        for w in (1, 2, 3, 8):
            parts = [shard(n, r, w) for r in range(w)]
            flat = [i for p in parts for i in p]
            assert flat == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        vals = max_over_ranks([1.0 + rank, 10.0 - rank])
        out.put((rank, vals, shard(48, rank, world)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == [2.0, 10.0] and res[1][1] == [2.0, 10.0]
    assert res[0][2] + res[1][2] == list(range(48))


def test_max_over_ranks_single_process():
    assert max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
