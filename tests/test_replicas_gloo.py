"""The multi-process path on CPU: two gloo ranks, the q-point sharding and the
max-over-ranks timing that bench.py uses with one process per GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from ecalj_b200.replicas import max_over_ranks, shard


def test_shard_covers_every_item_once():
    for n in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in shard(n, r, world)]
            assert got == list(range(n))
            sizes = [len(shard(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = list(shard(64, rank, world))
        ms = 10.0 + rank * 5.0                            # rank 1 is the slow one
        out[rank] = (len(mine), mine[0], max_over_ranks(ms, dist, "cpu"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == (32, 0, 15.0) and out[1] == (32, 32, 15.0)
    assert max_over_ranks(3.5) == 3.5                     # not distributed: the value itself
