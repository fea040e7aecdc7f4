"""Host logic of the multi-GPU path on CPU ranks (gloo): view sharding and the snapshot exchange.

On GPUs the exchange broadcasts into each GPU's own snapshot buffer over NCCL; here the same function runs on CPU
tensors with two gloo ranks.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cumulus3d_b200.multigpu import exchange_regions, owner_regions, shard


def test_shard_covers_views_once_and_balances():
    for n in [1, 5, 24, 48, 64]:
        for world in [1, 2, 3, 4, 8]:
            parts = [shard(n, r, world) for r in range(world)]
            flat = [v for p in parts for v in p]
            assert flat == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


def test_owner_regions_are_contiguous_blocks():
    sizes = [12, 12, 7, 7, 9]
    offs = list(np.concatenate([[0], np.cumsum(sizes)[:-1]]))
    regs = owner_regions(offs, sizes, 2)
    assert regs == [(0, 31), (31, 16)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        offs = list(np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int))
        buf = torch.zeros(int(sum(sizes)), dtype=torch.float32)
        for v in shard(len(sizes), rank, world):  # each rank writes only the depth maps of its own views
            buf[offs[v]:offs[v] + sizes[v]] = float(100 * v + 1)
        exchange_regions(buf, owner_regions(offs, sizes, world))
        want = torch.cat([torch.full((s,), float(100 * v + 1)) for v, s in enumerate(sizes)])
        q.put((rank, bool(torch.equal(buf, want))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_snapshot_exchange_two_gloo_ranks(world):
    sizes = [6, 6, 6, 4, 4]  # 5 views of uneven sizes, sharded 3 + 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(res[r] for r in range(world)), res
