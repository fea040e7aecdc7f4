"""Depth-map driver over a PatchMatch session: the schedule of ``compute_depth_maps``
(crates/dense/src/densify.rs:212-498) for callers of this engine.

* :func:`compute_depth_maps` — the reference's multi-scale flow through the host-state session API (run at the coarsest
  level from random init; per finer level: upsample → evaluate → restorer run → evaluate → per-pixel restorer choice;
  geometric rounds against snapshots; final median filter / filter / readout threshold).
* :func:`schedule_resident` — the same single-level schedule entirely on the device (states, snapshots, filter and
  readout stay in HBM), used by the benchmark's device-resident leg.
* :func:`build_pyramid`, :func:`num_levels`, :func:`readout` — host helpers restating upsample.rs:35-102 and
  densify.rs:441-454.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from .patchstereo import DepthSnapshot, KernelInput, LevelImage, PatchMatchSession, RunParams, ViewState


@dataclass
class Schedule:
    """LevelSchedule (crates/dense/src/params.rs:62-73) plus the multi-scale constants of DensifyOptions."""
    photometric_iters: int = 6
    restorer_random_init: bool = False
    geometric_rounds: int = 2
    geometric_iters: int = 2
    photometric_iters_upper: int = 3  # fast profile: 6 at level 0, 3 above (params.rs:496-503)
    jbu_sigma_spatial: float = 1.0
    jbu_sigma_color: float = 0.04
    restorer_threshold: float = 0.1

    def at(self, level: int) -> "Schedule":
        s = Schedule(**self.__dict__)
        if level > 0:
            s.photometric_iters = self.photometric_iters_upper
        return s


def num_levels(min_side: int, max_levels: int, min_size: int) -> int:
    """upsample.rs:35-44."""
    l, s = 1, min_side
    while l < max_levels and s // 2 >= min_size:
        s //= 2
        l += 1
    return l


def build_pyramid(gray: np.ndarray, k: Sequence[float], levels: int) -> List[LevelImage]:
    """u8 pyramid (upsample.rs:46-102): separable 3-tap Gaussian (σ = 0.5, clamped borders), 2×2 average, rounding
    to u8; f ← f/2, c ← (c + 0.5)/2 − 0.5.  Returns level 0 = coarsest."""
    g0 = np.float32(np.exp(np.float32(-1.0) / np.float32(2.0 * 0.25)))
    g = np.array([g0, 1.0, g0], np.float32)
    g = g / g.sum(dtype=np.float32)
    out = [LevelImage(np.ascontiguousarray(gray), tuple(float(x) for x in k))]
    cur = gray.astype(np.float32)
    kk = [float(x) for x in k]
    for _ in range(1, levels):
        h, w = cur.shape
        xp = np.pad(cur, ((0, 0), (1, 1)), mode="edge")
        tmp = g[0] * xp[:, :-2] + g[1] * xp[:, 1:-1] + g[2] * xp[:, 2:]
        yp = np.pad(tmp, ((1, 1), (0, 0)), mode="edge")
        b = g[0] * yp[:-2] + g[1] * yp[1:-1] + g[2] * yp[2:]
        nh, nw = h // 2, w // 2
        b = b[: 2 * nh, : 2 * nw]
        nxt = np.float32(0.25) * (b[0::2, 0::2] + b[0::2, 1::2] + b[1::2, 0::2] + b[1::2, 1::2])
        fl = np.floor(nxt)  # values are >= 0: round half away from zero = floor + (frac >= 0.5), exact in binary32
        q = np.clip(fl + (nxt - fl >= np.float32(0.5)), 0, 255).astype(np.uint8)
        kk = [kk[0] * 0.5, kk[1] * 0.5, (kk[2] + 0.5) * 0.5 - 0.5, (kk[3] + 0.5) * 0.5 - 0.5]
        out.append(LevelImage(q, tuple(kk)))
        cur = q.astype(np.float32)
    out.reverse()
    return out


def build_pyramid_device(gray: np.ndarray, k: Sequence[float], levels: int, device: int = 0) -> List[LevelImage]:
    """build_pyramid on the GPU (ps_build_pyramid): the same levels as :func:`build_pyramid`, coarsest first."""
    import ctypes as C
    from . import _lib
    g = np.ascontiguousarray(gray, np.uint8)
    h, w = g.shape
    sizes = [(w, h)]
    for _ in range(1, levels):
        sizes.append((sizes[-1][0] // 2, sizes[-1][1] // 2))
    outs = [np.empty((sh, sw), np.uint8) for (sw, sh) in reversed(sizes)]
    op = (C.c_void_p * levels)(*[o.ctypes.data for o in outs])
    ow, oh = (C.c_uint32 * levels)(), (C.c_uint32 * levels)()
    kin = (C.c_double * 4)(*[float(x) for x in k])
    ko = (C.c_double * (4 * levels))()
    rc = _lib.engine().ps_build_pyramid(device, g.ctypes.data, w, h, kin, levels, op, ow, oh, ko)
    if rc != _lib.PS_OK:
        raise _lib.PsError(rc, "ps_build_pyramid failed")
    return [LevelImage(outs[i], tuple(ko[4 * i:4 * i + 4])) for i in range(levels)]


DEFAULT_SEED = 0x005EED0FDE75  # DensifyOptions::base().seed (crates/dense/src/params.rs:423)


def fast_filter():
    """FilterParams with the fast profile's tuning (crates/dense/src/params.rs:452-459)."""
    from . import _lib
    f = _lib.default_filter()
    f.min_ncc, f.geom_max_cost, f.min_num_consistent, f.median_filter = 0.2, 0.5, 3, 0
    return f


def kernel_input(cams, gray: Sequence[np.ndarray], sources: Sequence[Sequence[int]],
                 ranges: Sequence[Optional[tuple]], *, pm=None, filt=None, seed: int = DEFAULT_SEED,
                 max_levels: int = 3, min_level_size: int = 64) -> KernelInput:
    """The KernelInput compute_depth_maps assembles (crates/dense/src/densify.rs:277-312): the level count from the
    smallest image side, every view's 8-bit pyramid (coarsest first), key = FNV-1a of the image name, its sources with
    their pair geometry (binary32 and binary64), the depth range ((1, 2) where the view observes no point).  pm
    defaults to PmParams::default() (the fast profile's window), filt to the fast profile's filter."""
    from . import _lib
    from .patchstereo import KernelView, PairGeometry
    from .scenes import fnv1a, pair_geometry
    min_side = min(min(c.width, c.height) for c in cams)
    nl = num_levels(min_side, max(max_levels, 1), max(min_level_size, 8))
    views = []
    for v, cam in enumerate(cams):
        p64 = np.stack([pair_geometry(cam, cams[j]) for j in sources[v]]) if sources[v] else np.zeros((0, 15))
        pairs = [PairGeometry(p[:9].astype(np.float32), p[9:12].astype(np.float32), p[12:15].astype(np.float32))
                 for p in p64]
        dmin, dmax = ranges[v] if ranges[v] is not None else (1.0, 2.0)
        views.append(KernelView(fnv1a(cam.name.encode()), build_pyramid(np.asarray(gray[v], np.uint8), cam.k, nl),
                                list(sources[v]), pairs, float(dmin), float(dmax), p64))
    return KernelInput(views, nl, pm if pm is not None else _lib.default_pm(),
                       filt if filt is not None else fast_filter(), seed)


def readout(states: Sequence[ViewState], counts: Sequence[np.ndarray], nsrc: Sequence[int],
            min_num_consistent: int) -> List[ViewState]:
    """Readout threshold (densify.rs:441-454): depth/normal zeroed where count < max(1, min(min_num_consistent, nsrc)).
    Returns new states (the inputs are unchanged); views are processed on a thread pool (numpy releases the GIL on
    whole-array operations)."""
    zero = np.float32(0.0)

    def one(args):
        s, c, n = args
        need = max(1, min(min_num_consistent, n))
        keep = (s.depth > 0) & (c >= need)
        return ViewState(s.width, s.height, np.where(keep, s.depth, zero), np.where(keep[..., None], s.normal, zero),
                         s.cost.copy(), None if s.prior is None else s.prior.copy())

    items = list(zip(states, counts, nsrc))
    if len(items) < 2:
        return [one(a) for a in items]
    with ThreadPoolExecutor(max_workers=min(len(items), os.cpu_count() or 1)) as ex:
        return list(ex.map(one, items))


def compute_depth_maps(session: PatchMatchSession, inp: KernelInput, views: Sequence[int],
                       sch: Schedule = Schedule(), weak_texture_prior: bool = False):
    """The multi-scale schedule of compute_depth_maps (densify.rs:350-454) for `views`.  Returns (raw states at the
    top level, filtered states, filter counts)."""
    nl = inp.num_levels
    top = nl - 1
    run_id = 0
    snap_id = 0

    def next_run():
        nonlocal run_id
        run_id += 1
        return run_id

    def snapshot(level, states):
        nonlocal snap_id
        snap_id += 1
        maps: List[Optional[np.ndarray]] = [None] * len(inp.views)
        for v, s in zip(views, states):
            maps[v] = s.depth.copy()
        return DepthSnapshot(snap_id, level, maps)

    def size(v, l):
        li = inp.views[v].levels[l]
        return li.width, li.height

    states: List[ViewState] = []
    for level in range(nl):
        s = sch.at(level)
        use_prior = level > 0 and inp.pm.weak_texture_var > 0.0 and weak_texture_prior
        if level == 0:
            states = [ViewState.new(*size(v, 0)) for v in views]
            session.run(views, states, RunParams(level, False, True, s.photometric_iters, next_run(), False))
        else:
            up = session.upsample(inp, level, views, states, s.jbu_sigma_spatial, s.jbu_sigma_color)
            if use_prior:
                for u in up:
                    u.prior = np.ascontiguousarray(u.planes())
            c_init = session.evaluate(level, views, up, False, None)
            if s.restorer_random_init:
                photo = [ViewState.new(u.width, u.height) for u in up]
                for p, u in zip(photo, up):
                    p.prior = u.prior
            else:
                photo = [u.copy() for u in up]
            session.run(views, photo, RunParams(level, False, s.restorer_random_init, s.photometric_iters, next_run(),
                                                use_prior))
            c_photo = session.evaluate(level, views, photo, False, None)
            new = []
            for u, ph, ci, cp in zip(up, photo, c_init, c_photo):
                take = (u.depth <= 0.0) | ((ci - cp) > s.restorer_threshold)
                u.depth[take] = ph.depth[take]
                u.normal[take] = ph.normal[take]
                new.append(u)
            states = new
        for _ in range(s.geometric_rounds):
            snap = snapshot(level, states)
            session.run(views, states, RunParams(level, True, False, s.geometric_iters, next_run(), use_prior), snap)
    for st in states:
        st.prior = None
    if inp.filter.median_filter:
        states = session.median_filter(inp, top, views, states)
    snap = snapshot(top, states)
    counts = session.filter(views, states, snap)
    nsrc = [len(inp.views[v].sources) for v in views]
    return states, readout(states, counts, nsrc, inp.filter.min_num_consistent), counts


def compute_depth_maps_resident(session: PatchMatchSession, inp: KernelInput, views: Sequence[int],
                                sch: Schedule = Schedule(), weak_texture_prior: bool = False,
                                graph: bool = True) -> List[ViewState]:
    """compute_depth_maps on the device (ps_schedule_multiscale): the same schedule, no host round trips, one graph
    launch.  Returns the filtered states (readout) of the top level."""
    if sch.restorer_random_init:
        raise ValueError("the device driver implements the restorer without random init (the fast profile)")
    session.schedule_multiscale(views, sch.photometric_iters, sch.photometric_iters_upper, sch.geometric_rounds,
                                sch.geometric_iters, sch.jbu_sigma_spatial, sch.jbu_sigma_color,
                                sch.restorer_threshold, weak_texture_prior, 1, graph)
    return session.readout_download(inp.num_levels - 1, views)


def schedule_host(session: PatchMatchSession, inp: KernelInput, views: Sequence[int], photometric_iters: int,
                  geometric_rounds: int, geometric_iters: int):
    """Single-level schedule through the host-state API (every call copies states in and out, as the reference's
    session does).  Returns (raw states, filtered states, counts)."""
    level = 0
    states = [ViewState.new(inp.views[v].levels[0].width, inp.views[v].levels[0].height) for v in views]
    run_id = 1
    session.run(views, states, RunParams(level, False, True, photometric_iters, run_id))
    snap_id = 0
    for _ in range(geometric_rounds):
        snap_id += 1
        run_id += 1
        maps: List[Optional[np.ndarray]] = [None] * len(inp.views)
        for v, s in zip(views, states):
            maps[v] = s.depth
        session.run(views, states, RunParams(level, True, False, geometric_iters, run_id),
                    DepthSnapshot(snap_id, level, maps))
    snap_id += 1
    maps = [None] * len(inp.views)
    for v, s in zip(views, states):
        maps[v] = s.depth
    counts = session.filter(views, states, DepthSnapshot(snap_id, level, maps))
    nsrc = [len(inp.views[v].sources) for v in views]
    return states, readout(states, counts, nsrc, inp.filter.min_num_consistent), counts


def schedule_resident(session: PatchMatchSession, views: Sequence[int], photometric_iters: int, geometric_rounds: int,
                      geometric_iters: int, level: int = 0, snap_base: int = 1_000_000) -> None:
    """Single-level schedule with every state on the device: photometric run from random init, geometric rounds against
    device-captured snapshots, filter, readout threshold.  Results stay resident (download with session.download /
    readout_resident)."""
    run_id = 1
    session.run_resident(views, RunParams(level, False, True, photometric_iters, run_id))
    for r in range(geometric_rounds):
        run_id += 1
        session.snapshot_capture(level, views, snap_base + 2 * r)
        session.run_resident(views, RunParams(level, True, False, geometric_iters, run_id))
    session.snapshot_capture(level, views, snap_base + 2 * geometric_rounds + 1)
    session.filter_resident(views, download=False)
    session.readout_resident(views, download=False)
