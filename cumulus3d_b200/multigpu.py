"""Multi-GPU execution of one depth-map job: views sharded over ranks, one exchange per geometric round.

PatchStereo runs are independent per reference view except for the geometric rounds, which read the previous
round's depth maps of the source views (crates/dense/src/densify.rs:411-422).  So one job shards by view
(contiguous blocks, one process per GPU) and the only collective is, before each geometric round and before the
filter, the exchange of depth snapshots: every rank broadcasts the maps of the views it owns, over NCCL, straight
into every other GPU's own snapshot buffer (never a peer-memory load in a kernel).  The exchange is written over
torch tensors so the same code runs on NCCL/GPU and on gloo/CPU in tests.
"""
from __future__ import annotations

from typing import Callable, List, Sequence

import numpy as np

from .patchstereo import DepthSnapshot, KernelInput, PatchMatchSession, RunParams, ViewState


def shard(n_views: int, rank: int, world: int) -> List[int]:
    """Contiguous view blocks whose sizes differ by at most one."""
    base, extra = divmod(n_views, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def owner_regions(offsets: Sequence[int], sizes: Sequence[int], world: int, shard_fn: Callable = shard):
    """Per rank: (start, length) in floats of its views' block in a buffer laid out by `offsets` (view order)."""
    out = []
    n = len(offsets)
    for r in range(world):
        vs = shard_fn(n, r, world)
        if not vs:
            out.append((0, 0))
            continue
        a, b = vs[0], vs[-1]
        assert all(offsets[v + 1] == offsets[v] + sizes[v] for v in vs[:-1]), "views of a block must be contiguous"
        out.append((offsets[a], offsets[b] + sizes[b] - offsets[a]))
    return out


def exchange_regions(buf, regions, group=None) -> None:
    """Broadcasts every rank's region of `buf` (a 1-D tensor) from its owner to all ranks, in rank order."""
    import torch.distributed as dist
    for src, (start, length) in enumerate(regions):
        if length:
            dist.broadcast(buf[start:start + length], src=src, group=group)


class _DeviceArray:
    """__cuda_array_interface__ view of a device float buffer (so torch can wrap the engine's snapshot memory)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


class SnapshotExchange:
    """Runs a single-level schedule for this rank's views with the geometric-round snapshot exchange."""

    def __init__(self, session: PatchMatchSession, inp: KernelInput, world: int, rank: int, shard_fn=shard,
                 level: int = 0, group=None):
        import torch
        self.s, self.inp, self.world, self.rank, self.level, self.group = session, inp, world, rank, level, group
        n = len(inp.views)
        self.all_views = list(range(n))
        self.mine = shard_fn(n, rank, world)
        ptr, offs = session.snapshot_buffer(level)
        sizes = [v.levels[level].width * v.levels[level].height for v in inp.views]
        total = offs[-1] + sizes[-1]
        self.buf = torch.as_tensor(_DeviceArray(ptr, total), device=f"cuda:{torch.cuda.current_device()}")
        self.regions = owner_regions(offs, sizes, world, shard_fn)
        self.snap_id = 0

    def _snapshot(self):
        import torch
        self.snap_id += 1
        self.s.snapshot_capture(self.level, self.mine, 2_000_000 + self.snap_id)
        self.s.synchronize()
        exchange_regions(self.buf, self.regions, self.group)
        torch.cuda.synchronize()
        self.s.snapshot_mark(self.level, self.all_views, 2_000_000 + self.snap_id)

    def schedule(self, mine, photometric_iters: int, geometric_rounds: int, geometric_iters: int) -> None:
        run_id = 1
        self.s.run_resident(mine, RunParams(self.level, False, True, photometric_iters, run_id))
        for _ in range(geometric_rounds):
            run_id += 1
            self._snapshot()
            self.s.run_resident(mine, RunParams(self.level, True, False, geometric_iters, run_id))
        self._snapshot()
        self.s.filter_resident(mine, download=False)
        self.s.readout_resident(mine, download=False)

    def close(self):
        self.buf = None


def host_schedule_sharded(session: PatchMatchSession, inp: KernelInput, mine: Sequence[int], photometric_iters: int,
                          geometric_rounds: int, geometric_iters: int, world: int, rank: int, group=None):
    """The single-level schedule through the host-state ABI for this rank's views; depth maps of all views are
    exchanged through host-staged tensors before each geometric round and the filter."""
    import torch
    import torch.distributed as dist
    n = len(inp.views)
    sizes = [v.levels[0].width * v.levels[0].height for v in inp.views]
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    dev = f"cuda:{torch.cuda.current_device()}" if torch.cuda.is_available() else "cpu"
    states = [ViewState.new(inp.views[v].levels[0].width, inp.views[v].levels[0].height) for v in mine]
    run_id = 1
    session.run(mine, states, RunParams(0, False, True, photometric_iters, run_id))

    def snapshot(snap_id):
        buf = torch.zeros(int(sum(sizes)), dtype=torch.float32, device=dev)
        for v, s in zip(mine, states):
            buf[offs[v]:offs[v] + sizes[v]] = torch.from_numpy(s.depth.ravel()).to(dev)
        exchange_regions(buf, owner_regions(list(offs), sizes, world), group)
        host = buf.cpu().numpy()
        return DepthSnapshot(snap_id, 0, [host[offs[v]:offs[v] + sizes[v]] for v in range(n)])

    for r in range(geometric_rounds):
        run_id += 1
        session.run(mine, states, RunParams(0, True, False, geometric_iters, run_id), snapshot(r + 1))
    counts = session.filter(mine, states, snapshot(geometric_rounds + 1))
    return states, counts
