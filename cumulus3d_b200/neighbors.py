"""Neighbour (source) views and per-view depth ranges from sparse point tracks, on the GPU (ps_select_neighbors).

The engine's counterpart of ``PairStats::new``, ``PairStats::select_all`` / ``select_diverse`` and ``depth_ranges``
(crates/dense/src/neighbors.rs:44-186) as ``compute_depth_maps`` calls them (crates/dense/src/densify.rs:224-241):

* pair statistics: for every pair of distinct entries of every track, a shared count and the triangulation angle
  min(a, pi - a) at the point;
* selection: candidates with a 75th-percentile angle of at least ``min_triangulation_angle_deg`` (no test at 0) in
  descending shared count (ascending index on ties), at most ``num_views``; with ``diversity_decay`` < 1 the greedy
  choice that divides the count by ``decay`` per candidate already taken from the same baseline-azimuth sector;
* depth range: (0.75 x the 1 % depth, 1.25 x the 99 % depth) of the view's positive observation depths, None when the
  view observes nothing.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib


@dataclass
class SparseModel:
    """Sparse views and point tracks: views (n, 12) float64 = world -> camera rotation (row-major) then translation;
    xyz (p, 3) float64; track_offsets (p + 1,) uint32 into track_views (view indices)."""
    views: np.ndarray
    xyz: np.ndarray
    track_offsets: np.ndarray
    track_views: np.ndarray

    @staticmethod
    def from_tracks(rotations: Sequence[np.ndarray], translations: Sequence[np.ndarray], xyz: np.ndarray,
                    tracks: Sequence[Sequence[int]]) -> "SparseModel":
        views = np.array([np.concatenate([np.asarray(r, np.float64).ravel(), np.asarray(t, np.float64).ravel()])
                          for r, t in zip(rotations, translations)], np.float64).reshape(-1, 12)
        off = np.zeros(len(tracks) + 1, np.uint32)
        off[1:] = np.cumsum([len(t) for t in tracks])
        tv = np.array([v for t in tracks for v in t], np.uint32)
        return SparseModel(views, np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3)), off, tv)

    @property
    def num_views(self) -> int:
        return int(self.views.shape[0])


@dataclass
class NeighborParams:
    """NeighborOptions (crates/dense/src/params.rs:355-369)."""
    num_views: int = 10
    min_triangulation_angle_deg: float = 1.0
    direction_bins: int = 8
    diversity_decay: float = 1.0

    def c(self) -> _lib.NeighborParams:
        return _lib.NeighborParams(self.num_views, self.direction_bins, self.min_triangulation_angle_deg,
                                   self.diversity_decay)


@dataclass
class NeighborResult:
    sources: List[List[int]]
    depth_ranges: List[Optional[Tuple[float, float]]]
    pair_count: Optional[np.ndarray] = None    # (n, n) uint32, upper triangle (a < b) filled
    pair_angle75: Optional[np.ndarray] = None  # (n, n) float64, radians


def call(fn, model: SparseModel, params: NeighborParams, pair_stats: bool, *lead) -> NeighborResult:
    """Runs `fn` (ps_select_neighbors, or a function with its arguments after `lead`) on the model."""
    n = model.num_views
    views = (_lib.SparseView * max(n, 1))()
    for i in range(n):
        views[i].r[:] = [float(x) for x in model.views[i, :9]]
        views[i].t[:] = [float(x) for x in model.views[i, 9:12]]
    xyz = np.ascontiguousarray(model.xyz, np.float64)
    off = np.ascontiguousarray(model.track_offsets, np.uint32)
    tv = np.ascontiguousarray(model.track_views, np.uint32)
    if tv.size == 0:
        tv = np.zeros(1, np.uint32)
    src = np.empty((n, params.num_views), np.uint32)
    nsrc = np.empty(n, np.uint32)
    rng = np.empty((n, 2), np.float64)
    has = np.empty(n, np.uint8)
    pc = np.empty((n, n), np.uint32) if pair_stats else None
    pa = np.empty((n, n), np.float64) if pair_stats else None
    cp = params.c()
    rc = fn(*lead, views, n, xyz.ctypes.data, off.ctypes.data, tv.ctypes.data, len(off) - 1, C.byref(cp),
            src.ctypes.data, nsrc.ctypes.data, rng.ctypes.data, has.ctypes.data,
            pc.ctypes.data if pc is not None else None, pa.ctypes.data if pa is not None else None)
    if rc != _lib.PS_OK:
        raise _lib.PsError(rc, "neighbour selection failed")
    return NeighborResult([[int(v) for v in src[i, :nsrc[i]]] for i in range(n)],
                          [(float(rng[i, 0]), float(rng[i, 1])) if has[i] else None for i in range(n)], pc, pa)


def select_neighbors(model: SparseModel, params: NeighborParams = NeighborParams(), device: int = 0,
                     pair_stats: bool = False) -> NeighborResult:
    """Source views and depth ranges of every view of `model` on GPU `device`."""
    return call(_lib.engine().ps_select_neighbors, model, params, pair_stats, device)
