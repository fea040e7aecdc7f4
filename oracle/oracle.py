"""ctypes wrapper of the CPU oracle (oracle/_build/libps_oracle.so).  TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU-baseline / reference legs.  The engine
(cumulus3d_b200) never imports this module.  The entry points take the same C structs as include/patchstereo.h so a
test feeds identical inputs to the engine and to the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
from typing import List, Optional, Sequence

import numpy as np

from cumulus3d_b200 import _lib
from cumulus3d_b200.patchstereo import (CInput, DepthSnapshot, KernelInput, RunParams, ViewState, _views, c_snapshot,
                                        c_states)

PATH = pathlib.Path(__file__).resolve().parent / "_build" / "libps_oracle.so"
_o = None

_SV = C.POINTER(_lib.ViewState)
_KI = C.POINTER(_lib.KernelInput)
_U32P = C.POINTER(C.c_uint32)
_SNAP = C.POINTER(_lib.DepthSnapshot)


def lib() -> C.CDLL:
    global _o
    if _o is None:
        if not PATH.exists():
            raise RuntimeError(f"{PATH} is not built; run `make -C oracle`")
        o = C.CDLL(str(PATH))
        sig = {
            "oracle_run": (C.c_int, [_KI, _U32P, C.c_size_t, _SV, C.POINTER(_lib.RunParams), _SNAP, C.c_int]),
            "oracle_run_rows": (C.c_int, [_KI, _U32P, C.c_size_t, _SV, C.POINTER(_lib.RunParams), _SNAP, C.c_int,
                                          C.c_int, C.c_int]),
            "oracle_run_init": (C.c_int, [_KI, _U32P, C.c_size_t, _SV, C.POINTER(_lib.RunParams), _SNAP,
                                          C.POINTER(C.POINTER(C.c_float)), C.c_int, C.c_int, C.c_int]),
            "oracle_sweep": (C.c_int, [_KI, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]),
            "oracle_remove_speckles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float,
                                                 C.c_double, C.c_float, C.POINTER(C.c_uint64)]),
            "oracle_fuse": (C.c_int, [C.c_uint32, C.POINTER(_lib.FusionView), C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_void_p,
                                      C.POINTER(_lib.FusionParams), C.c_int, C.c_uint64, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                      C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "oracle_evaluate": (C.c_int, [_KI, C.c_uint32, _U32P, C.c_size_t, _SV, C.c_uint32, _SNAP,
                                          C.POINTER(C.POINTER(C.c_float)), C.c_int]),
            "oracle_filter": (C.c_int, [_KI, _U32P, C.c_size_t, _SV, _SNAP, C.POINTER(C.POINTER(C.c_uint8)), C.c_int]),
            "oracle_filter_rows": (C.c_int, [_KI, _U32P, C.c_size_t, _SV, _SNAP, C.POINTER(C.POINTER(C.c_uint8)),
                                             C.c_int, C.c_int, C.c_int]),
            "oracle_upsample": (C.c_int, [_KI, C.c_uint32, _U32P, C.c_size_t, _SV, C.c_float, C.c_float, _SV, C.c_int]),
            "oracle_median": (C.c_int, [_KI, C.c_uint32, _U32P, C.c_size_t, _SV, _SV, C.c_int]),
            "oracle_reeval_f64": (C.c_int, [_KI, C.c_uint32, _U32P, C.c_size_t, _SV, C.c_uint32, _SNAP,
                                            C.POINTER(C.POINTER(C.c_double)), C.c_int]),
            "oracle_select_neighbors": (C.c_int, [C.POINTER(_lib.SparseView), C.c_uint32, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_uint64, C.POINTER(_lib.NeighborParams), C.c_void_p,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
            "oracle_fill_holes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.POINTER(C.c_double), C.c_uint32, C.c_uint32, C.c_double, C.c_float,
                                            C.c_float, C.POINTER(C.c_uint64)]),
            "oracle_mix64": (C.c_uint64, [C.c_uint64]),
            "oracle_rng_state": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                              C.c_uint64]),
            "oracle_rng_next": (C.c_float, [C.POINTER(C.c_uint64)]),
            "oracle_hash_bytes": (C.c_uint64, [C.c_char_p, C.c_size_t]),
            "oracle_erf": (C.c_double, [C.c_double]),
            "oracle_emission_norm": (C.c_double, [C.c_double]),
            "oracle_emission": (C.c_double, [C.c_double, C.c_double]),
            "oracle_visibility_probability": (C.c_double, [C.c_double, C.c_double]),
            "oracle_triangulation_prior": (C.c_double, [C.c_double, C.c_double]),
            "oracle_incident_prior": (C.c_double, [C.c_double, C.c_double]),
            "oracle_resolution_prior": (C.c_double, [C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double]),
            "oracle_plane_transfer": (C.c_int, [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            "oracle_num_levels": (C.c_size_t, [C.c_size_t, C.c_size_t, C.c_size_t]),
            "oracle_pyramid_step": (None, [C.c_void_p, C.c_size_t, C.c_size_t, C.POINTER(C.c_double), C.c_void_p,
                                           C.POINTER(C.c_double)]),
            "oracle_expf": (C.c_float, [C.c_float]),
            "oracle_fuse_scored": (C.c_int, [C.c_uint32, C.POINTER(_lib.FusionView), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.POINTER(_lib.ScoreFusionParams),
                                             C.POINTER(_lib.FusionParams), C.c_int, C.c_uint64, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                             C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "oracle_smooth": (C.c_double, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_double, C.c_uint32, C.c_double,
                                           C.c_double, C.c_double, C.c_int]),
            "oracle_filter_visibility": (C.c_int64, [C.c_uint32, C.POINTER(_lib.FusionView), C.POINTER(C.c_uint32),
                                                     C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_void_p,
                                                     C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32,
                                                     C.c_uint32, C.c_double, C.c_void_p]),
            "oracle_exp64": (C.c_double, [C.c_double]),
            "oracle_acos64": (C.c_double, [C.c_double]),
            "oracle_sincosf": (None, [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
            "oracle_box_footprint_check": (C.c_int, [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, C.c_int,
                                                     C.POINTER(C.c_int)]),
        }
        for n, (r, a) in sig.items():
            f = getattr(o, n)
            f.restype, f.argtypes = r, a
        _o = o
    return _o


def _threads(threads: Optional[int]) -> int:
    return int(threads) if threads else (os.cpu_count() or 1)


def _chk(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with status {rc}")


def run(inp: KernelInput, views: Sequence[int], states: List[ViewState], p: RunParams,
        snapshot: Optional[DepthSnapshot] = None, threads: Optional[int] = None, rows=None,
        proposals: Optional[Sequence[np.ndarray]] = None) -> None:
    """PatchMatchSession::run restated on the CPU (states updated in place).  `rows` = (y0, y1) restricts the
    work to a band of rows (timing samples only).  With random_init = PS_INIT_PROPOSAL, `proposals[i]` (h, w, 4)
    f32 planes replace the random draw where d > 0 (the engine's learned init)."""
    ci, keep = CInput(inp), []
    rp = p.c()
    y0, y1 = rows if rows is not None else (0, 0)
    pp = None
    if proposals is not None:
        arrs = [np.ascontiguousarray(a, np.float32) for a in proposals]
        keep.append(arrs)
        pp = (C.POINTER(C.c_float) * max(len(arrs), 1))(*[a.ctypes.data_as(C.POINTER(C.c_float)) for a in arrs])
    _chk(lib().oracle_run_init(C.byref(ci.c), _views(views), len(views), c_states(states, keep), C.byref(rp),
                               c_snapshot(snapshot, keep), pp, _threads(threads), y0, y1), "run")


def sweep(inp: KernelInput, level: int, view: int, threads: Optional[int] = None,
          normal: Optional[Sequence[float]] = None) -> np.ndarray:
    """The plane-sweep network input of one view: (h, w, 48) uint16 bf16 bits (image, 32 costs, zeros)."""
    ci = CInput(inp)
    lv = inp.views[view].levels[level]
    h, w = lv.pixels.shape[:2]
    out = np.zeros((h, w, _lib.PS_NET_CH_IN), np.uint16)
    n = None if normal is None else np.ascontiguousarray(normal, np.float32)
    _chk(lib().oracle_sweep(C.byref(ci.c), level, view, out.ctypes.data, w, None if n is None else n.ctypes.data,
                            _threads(threads)), "sweep")
    return out


def evaluate(inp: KernelInput, level: int, views: Sequence[int], states: List[ViewState], geometric: bool = False,
             snapshot: Optional[DepthSnapshot] = None, threads: Optional[int] = None) -> List[np.ndarray]:
    ci, keep = CInput(inp), []
    outs = [np.empty((s.height, s.width), np.float32) for s in states]
    op = (C.POINTER(C.c_float) * max(len(outs), 1))(*[o.ctypes.data_as(C.POINTER(C.c_float)) for o in outs])
    _chk(lib().oracle_evaluate(C.byref(ci.c), level, _views(views), len(views), c_states(states, keep), int(geometric),
                               c_snapshot(snapshot, keep), op, _threads(threads)), "evaluate")
    return outs


def filter(inp: KernelInput, views: Sequence[int], states: List[ViewState], snapshot: DepthSnapshot,
           threads: Optional[int] = None, rows=None) -> List[np.ndarray]:
    """pm_filter restated: per-pixel consistent-source counts.  `rows` = (y0, y1) restricts the work to a band of
    rows (timing samples only; the other rows of the counts are 0)."""
    ci, keep = CInput(inp), []
    outs = [np.zeros((s.height, s.width), np.uint8) for s in states]
    op = (C.POINTER(C.c_uint8) * max(len(outs), 1))(*[o.ctypes.data_as(C.POINTER(C.c_uint8)) for o in outs])
    y0, y1 = rows if rows is not None else (0, 0)
    _chk(lib().oracle_filter_rows(C.byref(ci.c), _views(views), len(views), c_states(states, keep),
                                  c_snapshot(snapshot, keep), op, _threads(threads), int(y0), int(y1)), "filter")
    return outs


def upsample(inp: KernelInput, level: int, views: Sequence[int], low: List[ViewState], sigma_s: float, sigma_c: float,
             threads: Optional[int] = None) -> List[ViewState]:
    ci, keep = CInput(inp), []
    outs = [ViewState.new(inp.views[v].levels[level].width, inp.views[v].levels[level].height) for v in views]
    _chk(lib().oracle_upsample(C.byref(ci.c), level, _views(views), len(views), c_states(low, keep), sigma_s, sigma_c,
                               c_states(outs, keep), _threads(threads)), "upsample")
    return outs


def median(inp: KernelInput, level: int, views: Sequence[int], states: List[ViewState],
           threads: Optional[int] = None) -> List[ViewState]:
    ci, keep = CInput(inp), []
    outs = [ViewState.new(s.width, s.height) for s in states]
    _chk(lib().oracle_median(C.byref(ci.c), level, _views(views), len(views), c_states(states, keep),
                             c_states(outs, keep), _threads(threads)), "median")
    return outs


def reeval_f64(inp: KernelInput, level: int, views: Sequence[int], states: List[ViewState], geometric: bool = False,
               snapshot: Optional[DepthSnapshot] = None, threads: Optional[int] = None) -> List[np.ndarray]:
    """FP64 re-evaluation of the top-K cost of the given hypotheses."""
    ci, keep = CInput(inp), []
    outs = [np.empty((s.height, s.width), np.float64) for s in states]
    op = (C.POINTER(C.c_double) * max(len(outs), 1))(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
    _chk(lib().oracle_reeval_f64(C.byref(ci.c), level, _views(views), len(views), c_states(states, keep),
                                 int(geometric), c_snapshot(snapshot, keep), op, _threads(threads)), "reeval")
    return outs


class OracleSession:
    """The oracle behind the PatchMatchSession interface, so a driver (e.g. densify.compute_depth_maps) runs the
    same schedule on the CPU restatement as on the engine."""

    def __init__(self, inp: KernelInput, threads: Optional[int] = None):
        self.input, self.threads = inp, threads

    def run(self, views, states, p, snapshot=None):
        run(self.input, views, states, p, snapshot, self.threads)

    def evaluate(self, level, views, states, geometric=False, snapshot=None):
        return evaluate(self.input, level, views, states, geometric, snapshot, self.threads)

    def filter(self, views, states, snapshot):
        return filter(self.input, views, states, snapshot, self.threads)

    def upsample(self, inp, level, views, low, sigma_s, sigma_c):
        return upsample(self.input, level, views, low, sigma_s, sigma_c, self.threads)

    def median_filter(self, inp, level, views, states):
        outs = median(self.input, level, views, states, self.threads)
        for o, s in zip(outs, states):
            o.cost[...] = s.cost
        return outs


def remove_speckles(depth: np.ndarray, normal: np.ndarray, cost: np.ndarray, post) -> int:
    """remove_speckles restated (depth (h, w), normal (h, w, 3) updated in place); returns the erased pixel count."""
    assert depth.dtype == np.float32 and normal.dtype == np.float32 and depth.flags.c_contiguous
    h, w = depth.shape
    c = np.ascontiguousarray(cost, np.float32)
    n = C.c_uint64()
    _chk(lib().oracle_remove_speckles(depth.ctypes.data, normal.ctypes.data, c.ctypes.data, w, h,
                                      post.speckle_rel_depth, post.speckle_min_area_frac, post.speckle_keep_cost,
                                      C.byref(n)), "remove_speckles")
    return int(n.value)


def fill_holes(depth: np.ndarray, normal: np.ndarray, cost: np.ndarray, raw_cost: np.ndarray, gray: np.ndarray, k,
               post) -> int:
    """fill_holes restated (depth (h, w), normal (h, w, 3) and cost updated in place); gray (h, w) uint8, k the view's
    fx, fy, cx, cy.  Returns the filled pixel count."""
    assert depth.dtype == np.float32 and normal.dtype == np.float32 and cost.dtype == np.float32
    assert depth.flags.c_contiguous and normal.flags.c_contiguous and cost.flags.c_contiguous
    h, w = depth.shape
    rc_ = np.ascontiguousarray(raw_cost, np.float32)
    g = np.ascontiguousarray(gray, np.uint8)
    kk = (C.c_double * 4)(*[float(x) for x in k])
    n = C.c_uint64()
    _chk(lib().oracle_fill_holes(depth.ctypes.data, normal.ctypes.data, cost.ctypes.data, rc_.ctypes.data,
                                 g.ctypes.data, kk, w, h, post.fill_max_frac, post.fill_edge_step, post.fill_max_cost,
                                 C.byref(n)), "fill_holes")
    return int(n.value)


def fuse(cams, depths, normals, costs, images, views, params, threads: Optional[int] = None):
    """Consistency fusion restated.  cams: fusion.FusionCams of all views; depths/normals/costs/images per view (the
    images as the engine stores them: f32, u8 inputs divided by 255 in binary32); only `views` are used.  Returns a
    fusion.FusedCloud in the reference's point order."""
    from cumulus3d_b200.fusion import FusedCloud
    nv = len(depths)
    ws = (C.c_uint32 * nv)(*[d.shape[1] for d in depths])
    hs = (C.c_uint32 * nv)(*[d.shape[0] for d in depths])
    keep = [np.ascontiguousarray(a, np.float32) for a in list(depths) + list(normals) + list(costs) + list(images)]
    ptr = lambda arrs: (C.c_void_p * nv)(*[a.ctypes.data for a in arrs])
    dp, np_, cp, ip = (ptr(keep[i * nv:(i + 1) * nv]) for i in range(4))
    used = np.zeros(nv, np.uint8)
    used[list(views)] = 1
    cap = int(sum(int((d > 0).sum()) for d in depths)) + 1
    stride = int(params.consistency_num_images) + 1
    pos = np.empty((cap, 3), np.float32)
    nrm = np.empty((cap, 3), np.float32)
    col = np.empty((cap, 3), np.uint8)
    key = np.empty(cap, np.uint64)
    vc = np.empty(cap, np.uint8)
    vis = np.empty((cap, stride), np.uint16)
    n, r, vr = C.c_uint64(), C.c_uint64(), C.c_uint64()
    _chk(lib().oracle_fuse(nv, cams.table, ws, hs, dp, np_, cp, ip, used.ctypes.data, C.byref(params),
                           _threads(threads), cap, pos.ctypes.data, nrm.ctypes.data, col.ctypes.data, key.ctypes.data,
                           vc.ctypes.data, vis.ctypes.data, stride, C.byref(n), C.byref(r), C.byref(vr)), "fuse")
    k = int(n.value)
    out = FusedCloud(pos[:k], nrm[:k], col[:k], key[:k], vc[:k], vis[:k], int(r.value))
    out.visibility_removed = int(vr.value)
    return out


def filter_visibility(cams, depths, views, positions, visibility, check_views: int, min_violations: int,
                      tau: float):
    """filter_visibility (crates/dense/src/visibility.rs:106-151) on a bare cloud: cams a fusion.FusionCams (its
    overlap lists are the candidate order), depths one map per view (only `views` count), visibility one list of view
    indices per point.  Returns the keep mask (bool per point)."""
    nv = len(depths)
    ws = (C.c_uint32 * nv)(*[d.shape[1] for d in depths])
    hs = (C.c_uint32 * nv)(*[d.shape[0] for d in depths])
    keepalive = [np.ascontiguousarray(d, np.float32) for d in depths]
    dp = (C.c_void_p * nv)(*[a.ctypes.data for a in keepalive])
    used = np.zeros(nv, np.uint8)
    used[list(views)] = 1
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    n = pos.shape[0]
    stride = max([len(v) for v in visibility] + [1])
    vc = np.array([len(v) for v in visibility], np.uint8)
    vis = np.zeros((n, stride), np.uint16)
    for i, v in enumerate(visibility):
        vis[i, :len(v)] = v
    keep = np.empty(n, np.uint8)
    r = lib().oracle_filter_visibility(nv, cams.table, ws, hs, dp, used.ctypes.data, pos.ctypes.data, vc.ctypes.data,
                                       vis.ctypes.data, stride, n, check_views, min_violations, tau, keep.ctypes.data)
    if r < 0:
        raise RuntimeError("oracle_filter_visibility: invalid arguments")
    return keep.astype(bool)


def smooth(positions, normals, gsd: float, iterations: int, radius_gsd: float, sigma_range_gsd: float,
           normal_deg: float, threads: Optional[int] = None):
    """smooth_along_normals (crates/dense/src/smooth.rs:143-220) on a bare cloud: returns (new positions, the median
    absolute displacement of the last pass)."""
    pos = np.ascontiguousarray(positions, np.float32).copy()
    nrm = np.ascontiguousarray(normals, np.float32)
    assert pos.shape == nrm.shape and pos.ndim == 2 and pos.shape[1] == 3
    d = lib().oracle_smooth(pos.ctypes.data, nrm.ctypes.data, pos.shape[0], gsd, iterations, radius_gsd,
                            sigma_range_gsd, normal_deg, _threads(threads))
    return pos, float(d)


def fuse_scored(cams, depths, normals, costs, images, views, params, threads: Optional[int] = None, post=None):
    """Score fusion restated (fuse_scored, crates/dense/src/fusion_score.rs:314-435); inputs as for fuse.  With
    `post` (a FusionParams), its visibility filter and smoothing follow, as fuse_depth_maps_with runs them
    (crates/dense/src/densify.rs:535-556).  Returns a fusion.FusedCloud in the reference's point order: (view, pixel)
    ascending; `.visibility_removed` counts the points the filter removed."""
    from cumulus3d_b200.fusion import FusedCloud
    nv = len(depths)
    ws = (C.c_uint32 * nv)(*[d.shape[1] for d in depths])
    hs = (C.c_uint32 * nv)(*[d.shape[0] for d in depths])
    keep = [np.ascontiguousarray(a, np.float32) for a in list(depths) + list(normals) + list(costs) + list(images)]
    ptr = lambda arrs: (C.c_void_p * nv)(*[a.ctypes.data for a in arrs])
    dp, np_, cp, ip = (ptr(keep[i * nv:(i + 1) * nv]) for i in range(4))
    used = np.zeros(nv, np.uint8)
    used[list(views)] = 1
    cap = int(sum(int((d > 0).sum()) for d in depths)) + 1
    stride = int(params.num_neighbors) + 1
    pos = np.empty((cap, 3), np.float32)
    nrm = np.empty((cap, 3), np.float32)
    col = np.empty((cap, 3), np.uint8)
    key = np.empty(cap, np.uint64)
    vc = np.empty(cap, np.uint8)
    vis = np.empty((cap, stride), np.uint16)
    n, vr = C.c_uint64(), C.c_uint64()
    _chk(lib().oracle_fuse_scored(nv, cams.table, ws, hs, dp, np_, cp, ip, used.ctypes.data, C.byref(params),
                                  None if post is None else C.byref(post), _threads(threads), cap, pos.ctypes.data,
                                  nrm.ctypes.data, col.ctypes.data, key.ctypes.data, vc.ctypes.data, vis.ctypes.data,
                                  stride, C.byref(n), C.byref(vr)), "fuse_scored")
    k = int(n.value)
    out = FusedCloud(pos[:k], nrm[:k], col[:k], key[:k], vc[:k], vis[:k])
    out.visibility_removed = int(vr.value)
    return out


def select_neighbors(model, params, pair_stats: bool = False):
    """PairStats::new + select_all / select_diverse + depth_ranges (crates/dense/src/neighbors.rs:44-186) on the CPU;
    same inputs and outputs as cumulus3d_b200.neighbors.select_neighbors."""
    from cumulus3d_b200 import neighbors
    return neighbors.call(lib().oracle_select_neighbors, model, params, pair_stats)
