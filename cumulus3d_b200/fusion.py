"""Post-processing and consistency fusion of resident depth maps, and PLY output.

Drop-in for the stages after the readout threshold in the reference's densify driver: speckle removal
(crates/dense/src/postproc.rs:77-129, ``remove_speckles`` of PostParams, on by default), consistency fusion
(crates/dense/src/fusion.rs:219-459 with the defaults of crates/dense/src/params.rs:327-351) and the dense PLY
(crates/dense/src/densify.rs:143-153).  The kernels run on the session's resident readout planes
(``ps_postprocess_resident``, ``ps_fuse_resident``); this module builds the camera table and reads the cloud back.

Overlap order: the reference orders a view's fusion partners by shared sparse points (PairStats,
crates/dense/src/densify.rs:514-519); the synthetic scenes here have no sparse reconstruction, so partners are the
other views by camera-centre distance (ties by index), the same rule that picks their sources.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib


def default_post() -> _lib.PostParams:
    p = _lib.PostParams()
    _lib.engine().ps_post_params_default(C.byref(p))
    return p


def default_fusion(min_consistent_views: Optional[int] = None) -> _lib.FusionParams:
    p = _lib.FusionParams()
    _lib.engine().ps_fusion_params_default(C.byref(p))
    if min_consistent_views is not None:
        p.min_consistent_views = min_consistent_views
    return p


def default_score_fusion(**overrides) -> _lib.ScoreFusionParams:
    """ScoreFusionOptions::default() (crates/dense/src/fusion_score.rs:81-97); keyword arguments override fields
    (`lambda_` for the penalty coefficient, the field `lambda`)."""
    p = _lib.ScoreFusionParams()
    _lib.engine().ps_score_fusion_params_default(C.byref(p))
    for k, v in overrides.items():
        k = "lambda" if k == "lambda_" else k
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def median_interp(v: Sequence[float]) -> float:
    """median_in_place (crates/dense/src/math.rs:126-141): sorted, linear interpolation at 0.5·(n-1)."""
    if len(v) == 0:
        return 0.0
    s = sorted(float(x) for x in v)
    pos = 0.5 * (len(s) - 1)
    lo = int(np.floor(pos))
    hi = min(lo + 1, len(s) - 1)
    return s[lo] + (s[hi] - s[lo]) * (pos - lo)


def baselines(cams, sources: Sequence[Sequence[int]]) -> List[float]:
    """Representative baseline per view: median distance to its source centres (crates/dense/src/densify.rs:260-275)."""
    out = []
    for v, src in enumerate(sources):
        c = cams[v].center
        out.append(median_interp([float(np.sqrt(((c - cams[s].center) ** 2).sum())) for s in src]))
    return out


def overlap_lists(cams, limit: int = 12) -> List[List[int]]:
    ctr = np.array([c.center for c in cams])
    out = []
    for i in range(len(cams)):
        d = np.linalg.norm(ctr - ctr[i], axis=1)
        out.append([j for _, j in sorted((float(d[j]), j) for j in range(len(cams)) if j != i)][:limit])
    return out


class FusionCams:
    """ps_fusion_view table of every session view (keeps the overlap arrays alive)."""

    def __init__(self, cams, sources: Sequence[Sequence[int]], overlap: Optional[List[List[int]]] = None,
                 limit: int = 12, image_ids: Optional[Sequence[int]] = None):
        self.overlap = overlap if overlap is not None else overlap_lists(cams, limit)
        self.baselines = baselines(cams, sources)
        n = len(cams)
        self.table = (_lib.FusionView * max(n, 1))()
        self._keep = []
        for v, cam in enumerate(cams):
            f = self.table[v]
            f.k[:] = [float(x) for x in cam.k]
            f.r[:] = [float(x) for x in np.asarray(cam.r, np.float64).ravel()]
            f.t[:] = [float(x) for x in np.asarray(cam.t, np.float64).ravel()]
            f.baseline = self.baselines[v]
            f.image_id = int(image_ids[v]) if image_ids is not None else v
            ov = (C.c_uint32 * max(len(self.overlap[v]), 1))(*self.overlap[v])
            self._keep.append(ov)
            f.num_overlap = len(self.overlap[v])
            f.overlap = C.cast(ov, C.POINTER(C.c_uint32))


@dataclass
class FusedCloud:
    positions: np.ndarray  # (n, 3) f32
    normals: np.ndarray    # (n, 3) f32
    colors: np.ndarray     # (n, 3) u8
    keys: np.ndarray       # (n,) u64
    vis_counts: np.ndarray  # (n,) u8
    vis: np.ndarray        # (n, stride) u16, first vis_counts entries valid (ascending view indices)
    residual: int = 0      # the last `residual` points come from the second pass of leftover pixels

    def __len__(self) -> int:
        return int(self.positions.shape[0])

    def visibility(self, i: int) -> List[int]:
        return [int(x) for x in self.vis[i, : self.vis_counts[i]]]

    def num_residual(self) -> int:
        """DenseOutput::num_residual (crates/dense/src/densify.rs:155-158)."""
        return int(self.residual)

    def write_ply(self, path) -> None:
        """DenseOutput::write_ply (crates/dense/src/densify.rs:143-153): creates the parent folder."""
        _parent_dir(path)
        write_ply(path, self.positions, self.normals, self.colors)

    def write_residual_ply(self, path) -> bool:
        """DenseOutput::write_residual_ply (crates/dense/src/densify.rs:160-180): only the second-pass points; False
        without writing when there are none."""
        r = self.num_residual()
        if r == 0:
            return False
        _parent_dir(path)
        n = len(self)
        write_ply(path, self.positions[n - r:], self.normals[n - r:], self.colors[n - r:])
        return True


def _parent_dir(path) -> None:
    import pathlib
    parent = pathlib.Path(path).parent
    if str(parent):
        parent.mkdir(parents=True, exist_ok=True)


def write_ply(path, positions: np.ndarray, normals: Optional[np.ndarray] = None,
              colors: Optional[np.ndarray] = None) -> None:
    """Binary little-endian PLY in the reference's dense layout (x y z nx ny nz red green blue) via ps_write_ply."""
    pos = np.ascontiguousarray(positions, np.float32)
    nrm = None if normals is None else np.ascontiguousarray(normals, np.float32)
    col = None if colors is None else np.ascontiguousarray(colors, np.uint8)
    rc = _lib.engine().ps_write_ply(str(path).encode(), pos.shape[0], pos.ctypes.data,
                                    None if nrm is None else nrm.ctypes.data, None if col is None else col.ctypes.data)
    if rc != _lib.PS_OK:
        raise _lib.PsError(rc, f"ps_write_ply({path}) failed")


def fuse_depth_maps_with(session, level: int, views: Sequence[int], cams: FusionCams,
                         params: Optional[_lib.FusionParams] = None,
                         score: Optional[_lib.ScoreFusionParams] = None) -> FusedCloud:
    """fuse_depth_maps_with (crates/dense/src/densify.rs:505-556) on a session's resident readout planes: score fusion
    when `score` is given, else consistency fusion with `params`; the visibility filter and the smoothing of `params`
    follow either one.  `cams` carries the overlap lists (PairStats::select(v, lim, 0.0) in the reference, lim =
    score.num_neighbors or params.consistency_num_images)."""
    p = params if params is not None else default_fusion()
    if score is not None:
        session.fuse_scored_resident(level, views, cams, score, post=p)
    else:
        session.fuse_resident(level, views, cams, p)
    return session.fused_points()
