"""Multi-rank walk sharding and the global top-k exchange, on CPU with gloo."""

import math
import os
import socket

import pytest
import torch.multiprocessing as tmp

from dreams_rns.distributed import global_topk, merge_topk, shard_range


def test_shard_range_covers_everything():
    for n in (0, 1, 7, 4096, 4097):
        for world in (1, 2, 3, 8):
            got = [shard_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1


def test_merge_order_matches_device_topk():
    parts = [[(1.0, 5), (float("inf"), 9), (float("nan"), 0)], [(1.0, 2), (-2.0, 1), (3.0, 7)]]
    m = merge_topk(parts, 10)
    assert [i for _, i in m] == [9, 7, 2, 5, 1, 0]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, deltas, k, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a, b = shard_range(len(deltas), rank, world)
        local = sorted([(deltas[i], i) for i in range(a, b)], key=lambda t: (-t[0], t[1]))[:k]
        res = global_topk(local, k)
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_global_topk_two_ranks():
    import random
    rng = random.Random(3)
    deltas = [rng.uniform(-3, 1) for _ in range(257)]
    deltas[10] = deltas[200]          # a tie across the two shards
    k = 25
    mgr = tmp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    tmp.spawn(_worker, args=(2, port, deltas, k, out), nprocs=2, join=True)
    want = sorted([(d, i) for i, d in enumerate(deltas)], key=lambda t: (-t[0], t[1]))[:k]
    assert out[0] == want and out[1] == want
