"""Host logic of the multi-GPU path on CPU ranks (gloo): view sharding, the snapshot exchange, and the sharded
schedule itself.

On GPUs the exchange broadcasts into each GPU's own snapshot buffer over NCCL; here the same functions run on CPU
tensors with two gloo ranks, and the sharded schedule runs on the CPU oracle's sessions, so its result can be held
to the one-process schedule bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cumulus3d_b200.multigpu import exchange_views, owners, shard, shard_lpt


def test_shard_covers_views_once_and_balances():
    for n in [1, 5, 24, 48, 64]:
        for world in [1, 2, 3, 4, 8]:
            parts = [shard(n, r, world) for r in range(world)]
            flat = [v for p in parts for v in p]
            assert flat == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1


def test_lpt_shards_balance_mixed_sizes():
    """Longest processing time first on the mixed-size batch's four image sizes: every view once, and the largest
    rank load within 4/3 of the ideal (the contiguous blocks are far worse when sizes are sorted)."""
    sizes = [960 * 540, 1280 * 720, 1920 * 1080, 2048 * 1536]
    rng = np.random.default_rng(1)
    px = [sizes[i] for i in rng.integers(0, 4, 64)]
    for world in (2, 3, 4, 8):
        parts = shard_lpt(px, world)
        assert sorted(v for p in parts for v in p) == list(range(64))
        loads = [sum(px[v] for v in p) for p in parts]
        ideal = max(sum(px) / world, max(px))
        assert max(loads) <= 4 / 3 * ideal
        blocks = [sum(px[v] for v in shard(64, r, world)) for r in range(world)]
        assert max(loads) <= max(blocks)
    # 9 -> rank 0, 5 -> rank 1, 5 -> rank 1 (5 < 9), 1 -> rank 0 (9 < 10)
    assert owners(shard_lpt([5, 5, 9, 1], 2), 4) == [1, 1, 0, 0]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))


def _worker(rank, world, port, sizes, q):
    _init(rank, world, port)
    try:
        offs = list(np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(int))
        parts = shard_lpt(sizes, world)
        buf = torch.zeros(int(sum(sizes)), dtype=torch.float32)
        for v in parts[rank]:  # each rank writes only the depth maps of its own views
            buf[offs[v]:offs[v] + sizes[v]] = float(100 * v + 1)
        exchange_views(buf, offs, sizes, owners(parts, len(sizes)))
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


def _schedule_worker(rank, world, port, q):
    """One rank of the sharded single-level schedule on the CPU oracle: its LPT views, snapshots exchanged over gloo."""
    _init(rank, world, port)
    try:
        from cumulus3d_b200.multigpu import host_schedule_sharded, view_pixels
        from oracle import oracle
        wl = _schedule_workload()
        mine = shard_lpt(view_pixels(wl.input), world)[rank]
        sess = oracle.OracleSession(wl.input, threads=2)
        states, counts = host_schedule_sharded(sess, wl.input, mine, 2, 1, 1, world, rank)
        q.put((rank, mine, [(s.depth, s.normal, s.cost) for s in states], counts))
    finally:
        dist.destroy_process_group()


def _schedule_workload():
    from cumulus3d_b200 import scenes
    return scenes.workload_small(64, 48, views=5, window_radius=2, seed=17, iters=2, sources=3, positions=2)


def test_sharded_schedule_on_two_gloo_ranks_equals_one_process():
    """The single-level schedule (photometric run, a geometric round against exchanged snapshots, the filter) sharded
    over two ranks gives every view the bits of the one-process schedule: the exchange delivers every source's depth
    map before each geometric round and the filter."""
    from cumulus3d_b200 import densify
    from oracle import oracle
    wl = _schedule_workload()
    sess = oracle.OracleSession(wl.input, threads=2)
    want_states, _, want_counts = densify.schedule_host(sess, wl.input, wl.views, 2, 1, 1)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_schedule_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    seen = []
    for rank, mine, states, counts in got:
        assert mine and len(mine) == len(states) == len(counts)
        for v, (d, n, c), cnt in zip(mine, states, counts):
            np.testing.assert_array_equal(d, want_states[v].depth, err_msg=f"depth view {v} rank {rank}")
            np.testing.assert_array_equal(n, want_states[v].normal, err_msg=f"normal view {v}")
            np.testing.assert_array_equal(c, want_states[v].cost, err_msg=f"cost view {v}")
            np.testing.assert_array_equal(cnt, want_counts[v], err_msg=f"counts view {v}")
            seen.append(v)
    assert sorted(seen) == wl.views
