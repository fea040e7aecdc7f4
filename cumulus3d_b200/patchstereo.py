"""Python mirror of the reference's PatchMatch backend interface over the C ABI of libpatchstereo.so.

Names, argument meaning and error behaviour follow ``crates/dense/src/kernel.rs`` (types :80-189, traits :191-245) and
the CUDA backend ``crates/cuda/src/patchmatch.rs`` (CudaPatchMatch :91-298, Session :751-869):

* :class:`PatchMatchBackend` ≙ ``CudaPatchMatch`` (``name``, ``begin``);
* :class:`PatchMatchSession` ≙ ``Session`` (``run``, ``evaluate``, ``filter``, ``upsample``, ``median_filter``) plus the
  device-resident extension (``upload``, ``download``, ``run_resident``, ``snapshot_capture``, ``filter_resident``,
  ``readout_resident``);
* :class:`KernelInput`, :class:`KernelView`, :class:`LevelImage`, :class:`PairGeometry`, :class:`ViewState`,
  :class:`RunParams`, :class:`DepthSnapshot` mirror the reference structs field by field.

Errors raise :class:`PsError` carrying the ps_status code (``PS_EINVAL`` for bad sizes/parameters ≙
``Error::InvalidArgument``, ``PS_ECUDA`` ≙ ``Error::Invariant("CUDA: …")``, ``PS_ENODEV`` ≙ ``GpuError::NotAvailable``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import PsError

FP = C.POINTER(C.c_float)


def _fptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(FP)


@dataclass
class LevelImage:
    """LevelImage (kernel.rs:80-91); ``pixels`` is u8 (value/255) or f32 gray, row-major (h, w)."""
    pixels: np.ndarray
    k: Sequence[float]  # fx, fy, cx, cy (integer-centre convention)

    @property
    def width(self) -> int:
        return int(self.pixels.shape[1])

    @property
    def height(self) -> int:
        return int(self.pixels.shape[0])


@dataclass
class PairGeometry:
    """PairGeometry (kernel.rs:93-103): reference -> source rotation r (3×3), translation t, source centre."""
    r: np.ndarray
    t: np.ndarray
    center: np.ndarray


@dataclass
class KernelView:
    """KernelView (kernel.rs:105-120); ``pairs_f64`` (n×15 doubles) optionally drives the FP64 homography setup."""
    key: int
    levels: List[LevelImage]
    sources: List[int]
    pairs: List[PairGeometry]
    depth_min: float
    depth_max: float
    pairs_f64: Optional[np.ndarray] = None


@dataclass
class KernelInput:
    """KernelInput (kernel.rs:122-135)."""
    views: List[KernelView]
    num_levels: int
    pm: _lib.PmParams = field(default_factory=_lib.default_pm)
    filter: _lib.FilterParams = field(default_factory=_lib.default_filter)
    seed: int = 0x005E_ED0F_DE75  # DensifyOptions::base seed (params.rs:427)


@dataclass
class ViewState:
    """ViewState (kernel.rs:137-160): per-pixel depth, normal (h, w, 3), cost and optional prior (h, w, 4)."""
    width: int
    height: int
    depth: np.ndarray
    normal: np.ndarray
    cost: np.ndarray
    prior: Optional[np.ndarray] = None

    @staticmethod
    def new(width: int, height: int) -> "ViewState":
        """State with depth/normal 0 and cost 2 (ViewState::new, kernel.rs:155-159)."""
        return ViewState(width, height, np.zeros((height, width), np.float32),
                         np.zeros((height, width, 3), np.float32), np.full((height, width), 2.0, np.float32))

    def copy(self) -> "ViewState":
        return ViewState(self.width, self.height, self.depth.copy(), self.normal.copy(), self.cost.copy(),
                         None if self.prior is None else self.prior.copy())

    def planes(self) -> np.ndarray:
        return np.concatenate([self.normal, self.depth[..., None]], axis=-1)


@dataclass
class RunParams:
    """RunParams (kernel.rs:173-189).  random_init: False / True, or PS_INIT_PROPOSAL (2) for the learned init."""
    level: int
    geometric: bool
    random_init: int
    iterations: int
    run_id: int
    use_prior: bool = False

    def c(self) -> _lib.RunParams:
        return _lib.RunParams(self.level, int(self.geometric), int(self.random_init), self.iterations, self.run_id,
                              int(self.use_prior))


@dataclass
class DepthSnapshot:
    """DepthSnapshot (kernel.rs:162-171): maps[v] is view v's depth at ``level`` or None."""
    id: int
    level: int
    maps: List[Optional[np.ndarray]]


class CInput:
    """Marshals a KernelInput into the C structs, keeping every referenced buffer alive."""

    def __init__(self, inp: KernelInput):
        self.keep = []
        nv = len(inp.views)
        views = (_lib.KernelView * max(nv, 1))()
        for i, v in enumerate(inp.views):
            lv = (_lib.LevelImage * len(v.levels))()
            for l, li in enumerate(v.levels):
                px = np.ascontiguousarray(li.pixels)
                if px.dtype == np.uint8:
                    fmt = _lib.PS_IMAGE_U8
                elif px.dtype == np.float32:
                    fmt = _lib.PS_IMAGE_F32
                else:
                    raise PsError(_lib.PS_EINVAL, f"image dtype {px.dtype} (u8 or f32)")
                self.keep.append(px)
                lv[l].width, lv[l].height, lv[l].format, lv[l].stride = px.shape[1], px.shape[0], fmt, 0
                lv[l].pixels = px.ctypes.data
                lv[l].k[:] = [float(x) for x in li.k]
            self.keep.append(lv)
            n = len(v.sources)
            src = (C.c_uint32 * max(n, 1))(*v.sources)
            prs = (_lib.PairGeometry * max(n, 1))()
            for j, pg in enumerate(v.pairs):
                prs[j].r[:] = [float(x) for x in np.asarray(pg.r, np.float32).ravel()]
                prs[j].t[:] = [float(x) for x in np.asarray(pg.t, np.float32).ravel()]
                prs[j].center[:] = [float(x) for x in np.asarray(pg.center, np.float32).ravel()]
            self.keep += [src, prs]
            views[i].key = v.key & 0xFFFFFFFFFFFFFFFF
            views[i].levels = lv
            views[i].sources = src
            views[i].num_sources = n
            views[i].pairs = prs
            if v.pairs_f64 is not None:
                p64 = np.ascontiguousarray(v.pairs_f64, np.float64).reshape(n, 15)
                self.keep.append(p64)
                views[i].pairs_f64 = p64.ctypes.data_as(C.POINTER(C.c_double))
            views[i].depth_min = v.depth_min
            views[i].depth_max = v.depth_max
        self.keep.append(views)
        self.c = _lib.KernelInput(views, nv, inp.num_levels, inp.pm, inp.filter, inp.seed & 0xFFFFFFFFFFFFFFFF)


def c_states(states: Sequence[ViewState], keep: list):
    arr = (_lib.ViewState * max(len(states), 1))()
    for i, s in enumerate(states):
        for a in (s.depth, s.normal, s.cost):
            if a.dtype != np.float32 or not a.flags.c_contiguous:
                raise PsError(_lib.PS_EINVAL, "state arrays must be contiguous float32")
        arr[i].width, arr[i].height = s.width, s.height
        arr[i].depth, arr[i].normal, arr[i].cost = _fptr(s.depth), _fptr(s.normal), _fptr(s.cost)
        if s.prior is not None:
            p = np.ascontiguousarray(s.prior, np.float32)
            keep.append(p)
            arr[i].prior = _fptr(p)
    keep.append(arr)
    return arr


def c_snapshot(snap: Optional[DepthSnapshot], keep: list):
    if snap is None:
        return None
    n = len(snap.maps)
    maps = (FP * max(n, 1))()
    lens = (C.c_uint64 * max(n, 1))()
    for v, m in enumerate(snap.maps):
        if m is not None:
            a = np.ascontiguousarray(m, np.float32)
            keep.append(a)
            maps[v] = _fptr(a)
            lens[v] = a.size
    keep.append(maps)
    keep.append(lens)
    s = _lib.DepthSnapshot(snap.id, snap.level, n, maps, C.cast(lens, C.POINTER(C.c_uint64)))
    keep.append(s)
    return C.byref(s)


def _views(views: Sequence[int]):
    return (C.c_uint32 * max(len(views), 1))(*views)


def measure_fp32_peak(device: int = 0) -> float:
    """Measured FP32 FFMA throughput of the device in TFLOP/s."""
    t = C.c_double()
    rc = _lib.engine().ps_measure_fp32_peak(device, C.byref(t))
    if rc != _lib.PS_OK:
        raise PsError(rc, "fp32 probe failed")
    return t.value


class PatchMatchBackend:
    """CudaPatchMatch equivalent (crates/cuda/src/patchmatch.rs:91-298) on one B200."""

    def __init__(self, device: int = 0, math: str = "parity", max_batch: int = 64, batch_pixels: int = 0,
                 tuning: int = 0, checked: bool = False):
        self.lib = _lib.engine()
        o = _lib.Options()
        self.lib.ps_options_default(C.byref(o))
        o.math_mode = {"parity": _lib.PS_MATH_PARITY, "fast": _lib.PS_MATH_FAST}[math]
        o.max_batch = max_batch
        o.batch_pixels = batch_pixels
        o.tuning = tuning
        o.checked = int(bool(checked))
        self.device = device
        h = C.c_void_p()
        rc = self.lib.ps_backend_create(device, C.byref(o), C.byref(h))
        if rc != _lib.PS_OK:
            raise PsError(rc, f"no usable sm_100 device {device}")
        self.h = h

    def name(self) -> str:
        return self.lib.ps_backend_name(self.h).decode()

    def begin(self, inp: KernelInput) -> "PatchMatchSession":
        ci = CInput(inp)
        s = C.c_void_p()
        rc = self.lib.ps_begin(self.h, C.byref(ci.c), C.byref(s))
        if rc != _lib.PS_OK:
            raise PsError(rc, self.lib.ps_backend_last_error(self.h).decode())
        return PatchMatchSession(self, s, inp)

    def inject_failure(self, kind: int, after: int = 0) -> None:
        """Arms one host-side failure (ps_backend_inject_failure): after `after` more operations of `kind`
        (_lib.PS_INJECT_DEVICE_ALLOC or PS_INJECT_UPLOAD) succeed, the next one fails; PS_INJECT_NONE disarms.
        PS_INJECT_CHECK_PROBE (checked backends): the next synchronising call fails with PS_EFAULT from the kernels'
        own bounds test of one out-of-range index (no access is made)."""
        rc = self.lib.ps_backend_inject_failure(self.h, kind, after)
        if rc != _lib.PS_OK:
            raise PsError(rc, "ps_backend_inject_failure")

    def close(self):
        if self.h:
            self.lib.ps_backend_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PatchMatchSession:
    """Session equivalent (crates/cuda/src/patchmatch.rs:751-869); use as a context manager or call close()."""

    def __init__(self, be: PatchMatchBackend, h, inp: KernelInput):
        self.be, self.lib, self.h, self.input = be, be.lib, h, inp

    def _check(self, rc: int):
        if rc != _lib.PS_OK:
            raise PsError(rc, self.lib.ps_last_error(self.h).decode())

    def _size(self, v: int, level: int):
        li = self.input.views[v].levels[level]
        return li.width, li.height

    # ---- PatchMatchSession ------------------------------------------------------------------------------------
    def run(self, views: Sequence[int], states: List[ViewState], p: RunParams,
            snapshot: Optional[DepthSnapshot] = None) -> None:
        keep = []
        cs = c_states(states, keep)
        rp = p.c()
        self._check(self.lib.ps_run(self.h, _views(views), len(views), cs, C.byref(rp), c_snapshot(snapshot, keep)))

    def evaluate(self, level: int, views: Sequence[int], states: List[ViewState], geometric: bool = False,
                 snapshot: Optional[DepthSnapshot] = None) -> List[np.ndarray]:
        keep = []
        cs = c_states(states, keep)
        outs = [np.empty((s.height, s.width), np.float32) for s in states]
        op = (FP * max(len(outs), 1))(*[_fptr(o) for o in outs])
        self._check(self.lib.ps_evaluate(self.h, level, _views(views), len(views), cs, int(geometric),
                                         c_snapshot(snapshot, keep), op))
        return outs

    def filter(self, views: Sequence[int], states: List[ViewState], snapshot: DepthSnapshot) -> List[np.ndarray]:
        keep = []
        cs = c_states(states, keep)
        outs = [np.empty((s.height, s.width), np.uint8) for s in states]
        op = (C.POINTER(C.c_uint8) * max(len(outs), 1))(*[o.ctypes.data_as(C.POINTER(C.c_uint8)) for o in outs])
        self._check(self.lib.ps_filter(self.h, _views(views), len(views), cs, c_snapshot(snapshot, keep), op))
        return outs

    def upsample(self, inp: KernelInput, level: int, views: Sequence[int], low: List[ViewState], sigma_s: float,
                 sigma_c: float) -> List[ViewState]:
        keep = []
        cl = c_states(low, keep)
        outs = [ViewState.new(*self._size(v, level)) for v in views]
        co = c_states(outs, keep)
        self._check(self.lib.ps_upsample(self.h, level, _views(views), len(views), cl, sigma_s, sigma_c, co))
        return outs

    def median_filter(self, inp: KernelInput, level: int, views: Sequence[int],
                      states: List[ViewState]) -> List[ViewState]:
        keep = []
        ci = c_states(states, keep)
        outs = [ViewState.new(*self._size(v, level)) for v in views]
        co = c_states(outs, keep)
        self._check(self.lib.ps_median_filter(self.h, level, _views(views), len(views), ci, co))
        for o, s in zip(outs, states):
            o.cost[...] = s.cost
        return outs

    # ---- device-resident extension ----------------------------------------------------------------------------
    def upload(self, level: int, views: Sequence[int], states: List[ViewState]) -> None:
        keep = []
        self._check(self.lib.ps_state_upload(self.h, level, _views(views), len(views), c_states(states, keep)))

    def download(self, level: int, views: Sequence[int]) -> List[ViewState]:
        keep = []
        outs = [ViewState.new(*self._size(v, level)) for v in views]
        self._check(self.lib.ps_state_download(self.h, level, _views(views), len(views), c_states(outs, keep)))
        return outs

    def run_resident(self, views: Sequence[int], p: RunParams) -> None:
        rp = p.c()
        self._check(self.lib.ps_run_resident(self.h, _views(views), len(views), C.byref(rp)))

    def snapshot_capture(self, level: int, views: Sequence[int], snap_id: int, keep_others: bool = False) -> None:
        self._check(self.lib.ps_snapshot_capture(self.h, level, _views(views), len(views), snap_id, int(keep_others)))

    def snapshot_buffer(self, level: int):
        """(device pointer, per-view offsets in floats) of the level's snapshot buffer."""
        ptr = C.c_void_p()
        offs = (C.c_uint64 * max(len(self.input.views), 1))()
        self._check(self.lib.ps_snapshot_buffer(self.h, level, C.byref(ptr), offs))
        return int(ptr.value or 0), [int(offs[i]) for i in range(len(self.input.views))]

    def snapshot_mark(self, level: int, views: Sequence[int], snap_id: int) -> None:
        self._check(self.lib.ps_snapshot_mark(self.h, level, _views(views), len(views), snap_id))

    def filter_resident(self, views: Sequence[int], download: bool = True) -> Optional[List[np.ndarray]]:
        if not download:
            self._check(self.lib.ps_filter_resident(self.h, _views(views), len(views), None))
            return None
        outs = []
        for v in views:
            w, h = self._size(v, self._snap_level_guess())
            outs.append(np.empty((h, w), np.uint8))
        op = (C.POINTER(C.c_uint8) * max(len(outs), 1))(*[o.ctypes.data_as(C.POINTER(C.c_uint8)) for o in outs])
        self._check(self.lib.ps_filter_resident(self.h, _views(views), len(views), op))
        return outs

    def _snap_level_guess(self) -> int:
        return self.input.num_levels - 1

    def readout_resident(self, views: Sequence[int], download: bool = True) -> Optional[List[ViewState]]:
        if not download:
            self._check(self.lib.ps_readout_resident(self.h, _views(views), len(views), None))
            return None
        keep = []
        lvl = self._snap_level_guess()
        outs = [ViewState.new(*self._size(v, lvl)) for v in views]
        self._check(self.lib.ps_readout_resident(self.h, _views(views), len(views), c_states(outs, keep)))
        return outs

    def schedule_resident(self, views: Sequence[int], photometric_iters: int, geometric_rounds: int,
                          geometric_iters: int, level: int = 0, run_id_base: int = 1, graph: bool = True,
                          proposal: bool = False) -> None:
        """The whole single-level schedule on resident states (asynchronous); with `graph`, one CUDA-graph launch.
        With `proposal`, the photometric run starts from the stored proposals (PS_INIT_PROPOSAL)."""
        sch = _lib.Schedule(level, photometric_iters, geometric_rounds, geometric_iters, run_id_base, int(graph),
                            _lib.PS_INIT_PROPOSAL if proposal else _lib.PS_INIT_RANDOM)
        self._check(self.lib.ps_schedule_resident(self.h, _views(views), len(views), C.byref(sch)))

    # ---- post-processing and fusion ----------------------------------------------------------------------------
    def postprocess_resident(self, level: int, views: Sequence[int], post=None, count: bool = True,
                             intrinsics=None, filled: bool = False):
        """Speckle removal and (when enabled) hole filling on the readout planes (PostParams; defaults of the
        reference when `post` is None).  `intrinsics`: (num_views, 4) float64 fx, fy, cx, cy of every session view
        (the full-precision DenseView::k), or None for the level's.  Returns the erased pixel count (None without
        `count`), or (erased, filled) with `filled`."""
        from .fusion import default_post
        p = post if post is not None else default_post()
        n, f = C.c_uint64(), C.c_uint64()
        kp = None
        if intrinsics is not None:
            k = np.ascontiguousarray(intrinsics, np.float64).reshape(-1, 4)
            kp = k.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.ps_postprocess_resident(self.h, level, _views(views), len(views), C.byref(p), kp,
                                                     C.byref(n) if count else None, C.byref(f) if filled else None))
        if filled:
            return int(n.value), int(f.value)
        return int(n.value) if count else None

    def readout_download(self, level: int, views: Sequence[int]) -> List[ViewState]:
        """The current readout planes (after post-processing) and costs, without recomputing the readout."""
        out = [ViewState.new(*self._size(v, level)) for v in views]
        keep = []
        self._check(self.lib.ps_readout_download(self.h, level, _views(views), len(views), c_states(out, keep)))
        return out

    def fuse_resident(self, level: int, views: Sequence[int], cams, params=None) -> int:
        """Consistency fusion of the readout planes of `views`; `cams` is a fusion.FusionCams of every view."""
        from .fusion import default_fusion
        p = params if params is not None else default_fusion()
        n, r = C.c_uint64(), C.c_uint64()
        self._check(self.lib.ps_fuse_resident(self.h, level, _views(views), len(views), cams.table, C.byref(p),
                                              C.byref(n), C.byref(r)))
        self._fused = (int(n.value), int(p.consistency_num_images) + 1)
        self.fused_residual = int(r.value)  # points added by the second pass (they come last)
        vr = C.c_uint64()
        self._check(self.lib.ps_fused_visibility_removed(self.h, C.byref(vr)))
        self.fused_visibility_removed = int(vr.value)
        return int(n.value)

    def fuse_scored_resident(self, level: int, views: Sequence[int], cams, params=None, post=None) -> int:
        """Score fusion (fuse_scored, crates/dense/src/fusion_score.rs:314-435) of the readout planes of `views`;
        `cams` is a fusion.FusionCams of every view.  `post` (a FusionParams) adds its visibility filter and smoothing
        after the fusion, as fuse_depth_maps_with does.  fused_points() then gives the points in (view, pixel)
        order."""
        from .fusion import default_score_fusion
        p = params if params is not None else default_score_fusion()
        n = C.c_uint64()
        self._check(self.lib.ps_fuse_scored_resident(self.h, level, _views(views), len(views), cams.table,
                                                     C.byref(p), None if post is None else C.byref(post),
                                                     C.byref(n)))
        self._fused = (int(n.value), int(p.num_neighbors) + 1)
        self.fused_residual = 0
        vr = C.c_uint64()
        self._check(self.lib.ps_fused_visibility_removed(self.h, C.byref(vr)))
        self.fused_visibility_removed = int(vr.value)
        return int(n.value)

    def fused_points(self):
        from .fusion import FusedCloud
        n, stride = getattr(self, "_fused", (0, 1))
        pos = np.empty((n, 3), np.float32)
        nrm = np.empty((n, 3), np.float32)
        col = np.empty((n, 3), np.uint8)
        key = np.empty(n, np.uint64)
        nv = np.empty(n, np.uint8)
        vis = np.empty((n, stride), np.uint16)
        self._check(self.lib.ps_fused_points(self.h, n, pos.ctypes.data, nrm.ctypes.data, col.ctypes.data,
                                             key.ctypes.data, nv.ctypes.data, vis.ctypes.data, stride))
        return FusedCloud(pos, nrm, col, key, nv, vis, getattr(self, "fused_residual", 0))

    def schedule_multiscale(self, views: Sequence[int], photometric_iters: int = 6, photometric_iters_upper: int = 3,
                            geometric_rounds: int = 2, geometric_iters: int = 2, jbu_sigma_spatial: float = 1.0,
                            jbu_sigma_color: float = 0.04, restorer_threshold: float = 0.1,
                            weak_texture_prior: bool = False, run_id_base: int = 1, graph: bool = True) -> None:
        """The multi-scale driver over every level on the device (asynchronous); results in the top level's readout
        planes (readout_download(top, views))."""
        m = _lib.MultiscaleSchedule(photometric_iters, photometric_iters_upper, geometric_rounds, geometric_iters,
                                    jbu_sigma_spatial, jbu_sigma_color, restorer_threshold, int(weak_texture_prior),
                                    run_id_base, int(graph))
        self._check(self.lib.ps_schedule_multiscale(self.h, _views(views), len(views), C.byref(m)))

    # ---- learned proposal (no reference counterpart) ----------------------------------------------------------
    def sweep_volume(self, level: int, view: int, out_ptr: int, row_pixels: int) -> None:
        """Writes the view's network input (bf16 NHWC, 48 channels) to device memory at `out_ptr` (asynchronous on
        the session stream)."""
        self._check(self.lib.ps_sweep_volume(self.h, level, view, C.c_void_p(out_ptr), row_pixels))

    def set_sweep_normals(self, normals: Optional[np.ndarray]) -> None:
        """(n_views, 3) plane-sweep normals in each camera frame, or None for fronto-parallel planes."""
        if normals is None:
            self._check(self.lib.ps_set_sweep_normals(self.h, None))
            return
        a = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        self._check(self.lib.ps_set_sweep_normals(self.h, a.ctypes.data))

    def propose(self, net, level: int, views: Sequence[int], conf_threshold: float = 0.15,
                count: bool = True) -> Optional[int]:
        """Sweep + network + decode into the session's proposal store; returns the number of proposed pixels."""
        n = C.c_uint64()
        self._check(self.lib.ps_propose(self.h, net.h, level, _views(views), len(views), conf_threshold,
                                        C.byref(n) if count else None))
        return int(n.value) if count else None

    def proposal_upload(self, level: int, views: Sequence[int], planes: Sequence[np.ndarray]) -> None:
        arrs = [np.ascontiguousarray(a, np.float32) for a in planes]
        pp = (C.POINTER(C.c_float) * max(len(arrs), 1))(*[a.ctypes.data_as(C.POINTER(C.c_float)) for a in arrs])
        self._check(self.lib.ps_proposal_upload(self.h, level, _views(views), len(views), pp))

    def proposal_download(self, level: int, views: Sequence[int]):
        """Stored proposals: list of ((h, w, 4) planes, (h, w) confidences)."""
        outs = []
        for v in views:
            w, h = self._size(v, level)
            outs.append((np.empty((h, w, 4), np.float32), np.empty((h, w), np.float32)))
        pp = (C.POINTER(C.c_float) * max(len(outs), 1))(*[o[0].ctypes.data_as(C.POINTER(C.c_float)) for o in outs])
        cp = (C.POINTER(C.c_float) * max(len(outs), 1))(*[o[1].ctypes.data_as(C.POINTER(C.c_float)) for o in outs])
        self._check(self.lib.ps_proposal_download(self.h, level, _views(views), len(views), pp, cp))
        return outs

    def synchronize(self) -> None:
        self._check(self.lib.ps_synchronize(self.h))

    def launch_count(self) -> int:
        return int(self.lib.ps_launch_count(self.h))

    def stream(self) -> int:
        return int(self.lib.ps_session_stream(self.h) or 0)

    def set_profiling(self, on: bool = True) -> None:
        self._check(self.lib.ps_set_profiling(self.h, int(on)))

    def kernel_stats(self, kind: int) -> dict:
        ms, n, w = C.c_double(), C.c_uint64(), C.c_uint64()
        self._check(self.lib.ps_kernel_stats(self.h, kind, C.byref(ms), C.byref(n), C.byref(w)))
        st = (C.c_uint64 * 8)()
        self._check(self.lib.ps_kernel_staged_stats(self.h, kind, st))
        return {"ms": ms.value, "launches": n.value, "ncc_windows": w.value, "staged_windows": st[0],
                "box_restages": st[1], "unstaged": {"bound": st[2], "wide": st[3], "tall": st[4], "few_lanes": st[5]},
                "skipped_windows": st[6]}

    def reset_stats(self) -> None:
        self._check(self.lib.ps_reset_stats(self.h))

    def close(self) -> None:
        if self.h:
            self.lib.ps_end(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
