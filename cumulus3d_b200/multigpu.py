"""Multi-GPU execution of one depth-map job: views sharded over ranks, one exchange per geometric round.

PatchStereo runs are independent per reference view except for the geometric rounds, which read the previous
round's depth maps of the source views (crates/dense/src/densify.rs:411-422).  So one job shards by view (one process
per GPU; views assigned by pixel count, longest processing time first, so ranks balance when view sizes differ) and
the only collective is, before each geometric round and before the filter, the exchange of depth snapshots: the owner
of every view broadcasts its map, over NCCL, straight into every other GPU's own snapshot buffer (never a peer-memory
load in a kernel).  The exchange is written over torch tensors so the same code runs on NCCL/GPU and on gloo/CPU in
tests.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np

from .patchstereo import DepthSnapshot, KernelInput, PatchMatchSession, RunParams, ViewState


def shard(n_views: int, rank: int, world: int) -> List[int]:
    """Contiguous view blocks whose sizes differ by at most one (for views of equal size)."""
    base, extra = divmod(n_views, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def shard_lpt(pixels: Sequence[int], world: int) -> List[List[int]]:
    """Longest processing time first: views in descending pixel count (ascending index on ties) each go to the rank
    with the fewest pixels so far (the lowest rank on ties).  Returns every rank's views in ascending order; the
    largest load is at most 4/3 of the optimum."""
    load = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for v in sorted(range(len(pixels)), key=lambda i: (-int(pixels[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(v)
        load[r] += int(pixels[v])
    return [sorted(p) for p in parts]


def owners(parts: Sequence[Sequence[int]], n_views: int) -> List[int]:
    """The owning rank of every view."""
    own = [-1] * n_views
    for r, vs in enumerate(parts):
        for v in vs:
            own[v] = r
    assert all(o >= 0 for o in own), "every view needs an owner"
    return own


def exchange_views(buf, offsets: Sequence[int], sizes: Sequence[int], owner: Sequence[int], group=None) -> None:
    """Broadcasts every view's block of `buf` (a 1-D tensor laid out by `offsets`) from its owner to all ranks, in
    view order (the same collective sequence on every rank)."""
    import torch.distributed as dist
    for v, (start, length) in enumerate(zip(offsets, sizes)):
        if length:
            dist.broadcast(buf[int(start):int(start) + int(length)], src=int(owner[v]), group=group)


class _DeviceArray:
    """__cuda_array_interface__ view of a device float buffer (so torch can wrap the engine's snapshot memory)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def view_pixels(inp: KernelInput, level: int = 0) -> List[int]:
    return [v.levels[level].width * v.levels[level].height for v in inp.views]


class SnapshotExchange:
    """Runs a single-level schedule for this rank's views with the geometric-round snapshot exchange."""

    def __init__(self, session: PatchMatchSession, inp: KernelInput, world: int, rank: int, level: int = 0,
                 group=None):
        import torch
        self.s, self.inp, self.world, self.rank, self.level, self.group = session, inp, world, rank, level, group
        n = len(inp.views)
        self.all_views = list(range(n))
        sizes = view_pixels(inp, level)
        parts = shard_lpt(sizes, world)
        self.mine = parts[rank]
        self.owner = owners(parts, n)
        ptr, offs = session.snapshot_buffer(level)
        total = offs[-1] + sizes[-1]
        self.buf = torch.as_tensor(_DeviceArray(ptr, total), device=f"cuda:{torch.cuda.current_device()}")
        self.offsets, self.sizes = list(offs), sizes
        self.snap_id = 0

    def _snapshot(self):
        import torch
        self.snap_id += 1
        self.s.snapshot_capture(self.level, self.mine, 2_000_000 + self.snap_id)
        self.s.synchronize()
        exchange_views(self.buf, self.offsets, self.sizes, self.owner, self.group)
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
    """The single-level schedule through the host-state ABI for this rank's views (`mine` = shard_lpt of the views'
    pixel counts, this rank's part); depth maps of all views are exchanged through host-staged tensors before each
    geometric round and the filter.  Returns (states, counts) of `mine`."""
    import torch
    n = len(inp.views)
    sizes = view_pixels(inp)
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    owner = owners(shard_lpt(sizes, world), n)
    assert [v for v in range(n) if owner[v] == rank] == sorted(mine), "mine must be this rank's shard_lpt part"
    dev = f"cuda:{torch.cuda.current_device()}" if torch.cuda.is_available() else "cpu"
    states = [ViewState.new(inp.views[v].levels[0].width, inp.views[v].levels[0].height) for v in mine]
    run_id = 1
    session.run(mine, states, RunParams(0, False, True, photometric_iters, run_id))

    def snapshot(snap_id):
        buf = torch.zeros(int(sum(sizes)), dtype=torch.float32, device=dev)
        for v, s in zip(mine, states):
            buf[offs[v]:offs[v] + sizes[v]] = torch.from_numpy(s.depth.ravel()).to(dev)
        exchange_views(buf, list(offs), sizes, owner, group)
        host = buf.cpu().numpy()
        return DepthSnapshot(snap_id, 0, [host[offs[v]:offs[v] + sizes[v]] for v in range(n)])

    for r in range(geometric_rounds):
        run_id += 1
        session.run(mine, states, RunParams(0, True, False, geometric_iters, run_id), snapshot(r + 1))
    counts = session.filter(mine, states, snapshot(geometric_rounds + 1))
    return states, counts
