"""Seeded synthetic aerial workloads for the PatchStereo engine.

The workloads stand in for real imagery (no dataset is named): terrain heightfields with value-noise albedo, rendered
by ``csrc/ps_synth.cpp`` through camera formations:

* ``workload_small``  — small scenes for parity tests (the oracle finishes in seconds);
* ``workload_c1``     — 640×480, 3-camera formation at 30 m, 40° off nadir, 10 m baseline, σ=0.01 noise, each view a
                        reference with the other two as sources, depth 25–60 m, 11×11 window, 5 iterations;
* ``workload_c2``     — same generator at 1920×1080, 3 cameras × 8 positions 5 m apart along the track (24 views),
                        4 nearest sources, 13×13 window, 6 photometric iterations + a geometric-consistency round
                        + the filter;
* ``workload_c3``     — 64 reference views of mixed sizes from 4 terrains, 2–8 sources each;
* ``workload_c5``     — 3840×2160, 3 × 16 positions, terrain + box structures of 3–15 m.

Geometry helpers restate ``pair_geometry`` (crates/dense/src/densify.rs:183-205, FP64) and the FNV-1a view key
(crates/dense/src/math.rs:31-39, used at crates/dense/src/densify.rs:301).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .patchstereo import KernelInput, KernelView, LevelImage, PairGeometry


class _SynthScene(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("relief", C.c_double), ("wavelength", C.c_double), ("cell", C.c_double),
                ("x0", C.c_double), ("y0", C.c_double), ("x1", C.c_double), ("y1", C.c_double),
                ("noise_sigma", C.c_double), ("num_boxes", C.c_int), ("box_hmin", C.c_double),
                ("box_hmax", C.c_double), ("box_smin", C.c_double), ("box_smax", C.c_double),
                ("albedo_scale", C.c_double)]


_synth = None


class _RefSceneConfig(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("focal", C.c_double), ("grid_x", C.c_int),
                ("grid_y", C.c_int), ("spacing", C.c_double), ("altitude", C.c_double), ("seed", C.c_uint64),
                ("num_points", C.c_int), ("num_boxes", C.c_int), ("boxes", (C.c_double * 6) * 8)]


def _synth_lib():
    global _synth
    if _synth is None:
        if not _lib.SYNTH_PATH.exists():
            raise RuntimeError(f"{_lib.SYNTH_PATH} is not built; run `python -m cumulus3d_b200.build`")
        _synth = C.CDLL(str(_lib.SYNTH_PATH))
        _synth.synth_render.restype = C.c_int
        _synth.synth_render.argtypes = [C.POINTER(_SynthScene), C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_void_p]
        _synth.synth_reference_scene.restype = C.c_int
        _synth.synth_reference_scene.argtypes = [C.POINTER(_RefSceneConfig), C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.POINTER(C.c_int)]
    return _synth


def fnv1a(b: bytes) -> int:
    """hash_bytes (crates/dense/src/math.rs:31-39)."""
    h = 0xCBF29CE484222325
    for x in b:
        h ^= x
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


@dataclass
class Camera:
    name: str
    k: Tuple[float, float, float, float]  # fx, fy, cx, cy (integer-centre convention)
    r: np.ndarray  # world -> camera rotation (3×3, float64)
    t: np.ndarray  # world -> camera translation
    width: int
    height: int

    @property
    def center(self) -> np.ndarray:
        return -self.r.T @ self.t


def formation(width: int, height: int, positions: int, *, baseline: float = 10.0, spacing: float = 5.0,
              altitude: float = 30.0, pitch_deg: float = 40.0, hfov_deg: float = 60.0, cams_per_row: int = 3,
              prefix: str = "view", y0: float = 0.0) -> List[Camera]:
    """Cameras side by side (cross-track, `baseline` apart) at `altitude`, optical axis `pitch_deg` off nadir toward
    the track direction (+y); `positions` formation stations `spacing` apart along +y."""
    f = (width / 2.0) / math.tan(math.radians(hfov_deg) / 2.0)
    k = (f, f, (width - 1) / 2.0, (height - 1) / 2.0)
    p = math.radians(pitch_deg)
    zc = np.array([0.0, math.sin(p), -math.cos(p)])
    xc = np.array([1.0, 0.0, 0.0])
    yc = np.cross(zc, xc)
    r = np.stack([xc, yc, zc])
    cams = []
    for s in range(positions):
        for c in range(cams_per_row):
            ctr = np.array([(c - (cams_per_row - 1) / 2.0) * baseline, y0 + s * spacing, altitude])
            cams.append(Camera(f"{prefix}_p{s:02d}_c{c}.png", k, r.copy(), -r @ ctr, width, height))
    return cams


def _extent(cams: Sequence[Camera], zmin: float = -1.0) -> Tuple[float, float, float, float]:
    pts = []
    for cam in cams:
        fx, fy, cx, cy = cam.k
        for (u, v) in [(0, 0), (cam.width - 1, 0), (0, cam.height - 1), (cam.width - 1, cam.height - 1)]:
            d = cam.r.T @ np.array([(u - cx) / fx, (v - cy) / fy, 1.0])
            c = cam.center
            t = (c[2] - zmin) / max(-d[2], 1e-6)
            pts.append(c + t * d)
            pts.append(c)
    pts = np.array(pts)
    return pts[:, 0].min() - 5, pts[:, 1].min() - 5, pts[:, 0].max() + 5, pts[:, 1].max() + 5


def render(cams: Sequence[Camera], seed: int, *, relief: float = 8.0, wavelength: float = 24.0, cell: float = 0.1,
           noise_sigma: float = 0.01, boxes: int = 0, box_h: Tuple[float, float] = (3.0, 15.0),
           box_s: Tuple[float, float] = (4.0, 12.0), with_gt: bool = True,
           extent: Optional[Tuple[float, float, float, float]] = None):
    """Renders every camera (all must share width/height).  Returns images (n, h, w) f32 and, with `with_gt`,
    ground-truth depth (n, h, w) and normals (n, h, w, 3)."""
    w, h = cams[0].width, cams[0].height
    assert all(c.width == w and c.height == h for c in cams)
    x0, y0, x1, y1 = extent if extent is not None else _extent(cams)
    sc = _SynthScene(seed, relief, wavelength, cell, x0, y0, x1, y1, noise_sigma, boxes, box_h[0], box_h[1],
                     box_s[0], box_s[1], 1.0)
    n = len(cams)
    cam = np.zeros((n, 16), np.float64)
    for i, c in enumerate(cams):
        cam[i, :4] = c.k
        cam[i, 4:13] = c.r.ravel()
        cam[i, 13:] = c.t
    img = np.empty((n, h, w), np.float32)
    dep = np.empty((n, h, w), np.float32) if with_gt else None
    nrm = np.empty((n, h, w, 3), np.float32) if with_gt else None
    rc = _synth_lib().synth_render(C.byref(sc), cam.ctypes.data_as(C.POINTER(C.c_double)), n, w, h, img.ctypes.data,
                                   dep.ctypes.data if with_gt else None, nrm.ctypes.data if with_gt else None)
    if rc != 0:
        raise RuntimeError("synth_render failed")
    return img, dep, nrm


def up_normals(cams: Sequence[Camera], up=(0.0, 0.0, 1.0)) -> np.ndarray:
    """The world's up direction in each camera frame (R · up), turned to face the camera: (n_views, 3) f32, for the
    plane sweep of the learned proposal (its planes then follow the ground's tilt)."""
    out = np.zeros((len(cams), 3), np.float32)
    for i, c in enumerate(cams):
        n = np.asarray(c.r, np.float64) @ np.asarray(up, np.float64)
        n = n / np.linalg.norm(n)
        out[i] = -n if n[2] > 0 else n
    return out


def pair_geometry(ref: Camera, src: Camera) -> np.ndarray:
    """Reference -> source relative geometry in FP64 (crates/dense/src/densify.rs:183-205): R = R_s R_rᵀ,
    t = t_s - R t_r, centre = -Rᵀ t.  Returns 15 doubles (r[9], t[3], center[3])."""
    rr = src.r @ ref.r.T
    t = src.t - rr @ ref.t
    c = -(rr.T @ t)
    return np.concatenate([rr.ravel(), t, c])


def nearest_sources(cams: Sequence[Camera], k: int) -> List[List[int]]:
    """The k nearest other cameras by centre distance (ties by index)."""
    ctr = np.array([c.center for c in cams])
    out = []
    for i in range(len(cams)):
        d = np.linalg.norm(ctr - ctr[i], axis=1)
        order = sorted((float(d[j]), j) for j in range(len(cams)) if j != i)
        out.append([j for _, j in order[:k]])
    return out


def sparse_model(cams: Sequence[Camera], gt_depth: np.ndarray, points_per_view: int = 4000, seed: int = 0,
                 rel_tol: float = 0.005):
    """Sparse points and tracks standing in for a structure-from-motion model: seeded pixels of every view
    back-projected through its ground-truth depth, each seen by every view whose ground-truth depth at the projection
    (nearest pixel) agrees within `rel_tol`; points seen by fewer than two views are dropped.  Tracks list their views
    in ascending order.  Returns a neighbors.SparseModel."""
    from .neighbors import SparseModel
    rng = np.random.default_rng(seed)
    pts = []
    for i, c in enumerate(cams):
        ys = rng.integers(0, c.height, points_per_view)
        xs = rng.integers(0, c.width, points_per_view)
        d = gt_depth[i][ys, xs].astype(np.float64)
        ok = d > 0
        ray = np.stack([(xs - c.k[2]) / c.k[0], (ys - c.k[3]) / c.k[1], np.ones(points_per_view)], -1)[ok]
        pts.append((ray * d[ok, None] - c.t) @ c.r)  # world = Rᵀ (camera point - t)
    X = np.concatenate(pts)
    vis = np.zeros((len(X), len(cams)), bool)
    for j, c in enumerate(cams):
        P = X @ c.r.T + c.t
        z = P[:, 2]
        zs = np.where(z > 0, z, 1.0)
        ui = np.rint(c.k[0] * P[:, 0] / zs + c.k[2]).astype(np.int64)
        vi = np.rint(c.k[1] * P[:, 1] / zs + c.k[3]).astype(np.int64)
        inside = (z > 0) & (ui >= 0) & (vi >= 0) & (ui < c.width) & (vi < c.height)
        dg = np.zeros(len(X))
        dg[inside] = gt_depth[j][vi[inside], ui[inside]]
        vis[:, j] = inside & (dg > 0) & (np.abs(z - dg) <= rel_tol * dg)
    keep = vis.sum(1) >= 2
    vis = vis[keep]
    off = np.zeros(len(vis) + 1, np.uint32)
    off[1:] = np.cumsum(vis.sum(1))
    views = np.array([np.concatenate([c.r.ravel(), c.t]) for c in cams], np.float64)
    return SparseModel(views, np.ascontiguousarray(X[keep]), off, np.nonzero(vis)[1].astype(np.uint32))


def to_gray8(img: np.ndarray) -> np.ndarray:
    """A rendered unit-range image as the 8-bit gray the reference's LevelImage holds (crates/dense/src/kernel.rs:80-91):
    round(255·v), clamped."""
    return np.clip(np.round(np.asarray(img, np.float64) * 255.0), 0, 255).astype(np.uint8)


def unit_plane(gray8: np.ndarray) -> np.ndarray:
    """The engine's f32 plane of an 8-bit image: the correctly rounded u/255 per pixel."""
    return (np.asarray(gray8, np.float64) / 255.0).astype(np.float32)


def kernel_input(cams: Sequence[Camera], images: Sequence[np.ndarray], sources: Sequence[Sequence[int]],
                 depth_range: Tuple[float, float], *, window_radius: int, window_step: int = 1, seed: int = 0x005EED0FDE75,
                 fast_filter: bool = True, ranges: Optional[Sequence[Tuple[float, float]]] = None,
                 gray8: bool = True) -> KernelInput:
    """Single-level KernelInput: each view's image (8-bit gray by default, as the reference takes it; f32 with
    gray8=False), its sources with f32 pairs (and the FP64 pairs)."""
    views = []
    for i, cam in enumerate(cams):
        p64 = np.stack([pair_geometry(cam, cams[j]) for j in sources[i]]) if sources[i] else np.zeros((0, 15))
        pairs = [PairGeometry(p[:9].astype(np.float32), p[9:12].astype(np.float32), p[12:15].astype(np.float32))
                 for p in p64]
        dr = ranges[i] if ranges is not None else depth_range
        img = to_gray8(images[i]) if gray8 and np.asarray(images[i]).dtype != np.uint8 else images[i]
        views.append(KernelView(fnv1a(cam.name.encode()), [LevelImage(img, cam.k)], list(sources[i]), pairs,
                                float(dr[0]), float(dr[1]), p64))
    pm = _lib.default_pm()
    pm.window_radius = window_radius
    pm.window_step = window_step
    fl = _lib.default_filter()
    if fast_filter:  # fast-profile filter tuning (crates/dense/src/params.rs:452-459)
        fl.min_ncc, fl.geom_max_cost, fl.min_num_consistent, fl.median_filter = 0.2, 0.5, 3, 0
    return KernelInput(views, 1, pm, fl, seed)


@dataclass
class Workload:
    name: str
    cams: List[Camera]
    images: np.ndarray
    gt_depth: Optional[np.ndarray]
    gt_normal: Optional[np.ndarray]
    input: KernelInput
    photometric_iters: int
    geometric_rounds: int
    geometric_iters: int

    @property
    def views(self) -> List[int]:
        return list(range(len(self.cams)))

    def pixels(self) -> int:
        return sum(c.width * c.height for c in self.cams)

    def iterations(self) -> int:
        return self.photometric_iters + self.geometric_rounds * self.geometric_iters


def workload_small(width: int = 96, height: int = 72, views: int = 3, window_radius: int = 3, window_step: int = 1,
                   seed: int = 7, iters: int = 2, geo_rounds: int = 0, geo_iters: int = 1, sources: int = 2,
                   positions: int = 1) -> Workload:
    """A small scene the oracle finishes in seconds (same generator, lower resolution)."""
    cams = formation(width, height, positions, prefix=f"small{seed}")[: max(views, 2)]
    img, dep, nrm = render(cams, seed)
    src = nearest_sources(cams, min(sources, len(cams) - 1))
    inp = kernel_input(cams, list(img), src, (25.0, 60.0), window_radius=window_radius, window_step=window_step)
    return Workload("small", cams, img, dep, nrm, inp, iters, geo_rounds, geo_iters)


def workload_c1(seed: int = 1) -> Workload:
    cams = formation(640, 480, 1, prefix="c1")
    img, dep, nrm = render(cams, seed)
    src = [[j for j in range(3) if j != i] for i in range(3)]
    inp = kernel_input(cams, list(img), src, (25.0, 60.0), window_radius=5, window_step=1)
    return Workload("c1_640x480_3views_w11_5it", cams, img, dep, nrm, inp, 5, 0, 0)


def workload_c2(seed: int = 2, with_gt: bool = True, views: Optional[int] = None) -> Workload:
    cams = formation(1920, 1080, 8, prefix="c2")
    if views is not None:
        cams = cams[:views]
    img, dep, nrm = render(cams, seed, with_gt=with_gt)
    src = nearest_sources(cams, 4)
    inp = kernel_input(cams, list(img), src, (25.0, 60.0), window_radius=6, window_step=1)
    return Workload("c2_1920x1080_24views_w13_6it_geo", cams, img, dep, nrm, inp, 6, 1, 2)


C3_SIZES = ((960, 540), (1280, 720), (1920, 1080), (2048, 1536))


def workload_c3(seed: int = 3, scenes_n: int = 4, per_scene: int = 16, with_gt: bool = False,
                sizes=C3_SIZES) -> Workload:
    """Batched uneven workload: `scenes_n` seeded terrains × `per_scene` reference views; every view's size is drawn
    uniformly from `sizes`, its source count uniformly from 2..8 (nearest cameras of its own scene), depth range
    20-80 m.  Cameras of one scene fly a 4-wide formation; all views run in one session."""
    rng = np.random.default_rng(seed)
    cams_all: List[Camera] = []
    images: List[np.ndarray] = []
    sources: List[List[int]] = []
    gts = []
    for sc in range(scenes_n):
        base = formation(1920, 1080, per_scene // 4, cams_per_row=4, prefix=f"c3s{sc}", spacing=6.0)
        picks = rng.integers(0, len(sizes), per_scene)
        cams = []
        for cam, k in zip(base, picks):
            w, h = sizes[k]
            f = (w / 2.0) / math.tan(math.radians(60.0) / 2.0)
            cams.append(Camera(cam.name, (f, f, (w - 1) / 2.0, (h - 1) / 2.0), cam.r, cam.t, w, h))
        ext = _extent(cams)
        imgs: List[Optional[np.ndarray]] = [None] * len(cams)
        for (w, h) in sorted({(c.width, c.height) for c in cams}):
            idx = [i for i, c in enumerate(cams) if (c.width, c.height) == (w, h)]
            img, dep, _ = render([cams[i] for i in idx], seed * 100 + sc, with_gt=with_gt, extent=ext)
            for j, i in enumerate(idx):
                imgs[i] = img[j]
        off = len(cams_all)
        near = nearest_sources(cams, len(cams) - 1)
        for i in range(len(cams)):
            k = int(rng.integers(2, 9))
            sources.append([off + j for j in near[i][:k]])
        cams_all += cams
        images += imgs
    inp = kernel_input(cams_all, images, sources, (20.0, 80.0), window_radius=6, window_step=1)
    return Workload("c3_64views_mixed_sizes_2to8_sources", cams_all, None, None, None, inp, 6, 1, 2)


def workload_c5(seed: int = 5, views: Optional[int] = None, with_gt: bool = False) -> Workload:
    cams = formation(3840, 2160, 16, prefix="c5")
    if views is not None:
        cams = cams[:views]
    img, dep, nrm = render(cams, seed, boxes=40, with_gt=with_gt)
    src = nearest_sources(cams, 5)
    inp = kernel_input(cams, list(img), src, (20.0, 60.0), window_radius=6, window_step=1)
    return Workload("c5_3840x2160_48views_boxes", cams, img, dep, nrm, inp, 2, 1, 1)


# ---------------------------------------------------------------------------------------------- reference test scene
# SynthConfig::default() (crates/dense/src/synthetic.rs:108-121).
REFERENCE_BOXES = (((-3.0, -2.0, 0.0), (1.0, 2.5, 4.0)), ((3.0, 2.0, 0.0), (6.0, 5.0, 2.0)))


@dataclass
class ReferenceScene:
    """The reference's synthetic accuracy scene: views in its order (name synth_{j}_{i}.png, image id = index + 1),
    8-bit gray images, ground-truth camera-z depth and camera-frame normals, and the sparse model."""
    cams: List[Camera]
    gray: np.ndarray       # (n, h, w) uint8
    gt_depth: np.ndarray   # (n, h, w) float32, 0 where the ray misses
    gt_normal: np.ndarray  # (n, h, w, 3) float32
    model: "object"        # neighbors.SparseModel
    boxes: Tuple[Tuple[Tuple[float, float, float], Tuple[float, float, float]], ...]

    @property
    def image_ids(self) -> List[int]:
        return [i + 1 for i in range(len(self.cams))]

    def surface_distance(self, p) -> float:
        """SynthScene::surface_distance (synthetic.rs:292-308): distance to the floor or the nearest box surface."""
        best = abs(p[2])
        for mn, mx in self.boxes:
            inside = all(mn[a] <= p[a] <= mx[a] for a in range(3))
            if inside:
                dd = min(min(p[a] - mn[a], mx[a] - p[a]) for a in range(3))
            else:
                q = [max(mn[a] - p[a], 0.0, p[a] - mx[a]) for a in range(3)]
                dd = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2])
            best = min(best, dd)
        return best

    def surface_distances(self, pts: np.ndarray) -> np.ndarray:
        """surface_distance of every row of pts (n, 3), vectorised."""
        p = np.asarray(pts, np.float64)
        best = np.abs(p[:, 2])
        for mn, mx in self.boxes:
            mn, mx = np.asarray(mn), np.asarray(mx)
            inside = np.all((p >= mn) & (p <= mx), axis=1)
            din = np.min(np.minimum(p - mn, mx - p), axis=1)
            q = np.maximum(np.maximum(mn - p, 0.0), p - mx)
            dout = np.sqrt((q * q).sum(1))
            best = np.minimum(best, np.where(inside, din, dout))
        return best


def reference_scene(width: int = 384, height: int = 288, focal: float = 300.0, grid=(3, 3), spacing: float = 3.0,
                    altitude: float = 20.0, boxes=REFERENCE_BOXES, seed: int = 11,
                    num_points: int = 3000) -> ReferenceScene:
    """make_scene(&SynthConfig) (crates/dense/src/synthetic.rs:190-290), rendered by csrc/ps_synth.cpp."""
    from .neighbors import SparseModel
    cfg = _RefSceneConfig(width, height, focal, grid[0], grid[1], spacing, altitude, seed, num_points, len(boxes))
    for b, (mn, mx) in enumerate(boxes):
        for a in range(3):
            cfg.boxes[b][a] = mn[a]
            cfg.boxes[b][3 + a] = mx[a]
    n = grid[0] * grid[1]
    cams = np.zeros((n, 16), np.float64)
    gray = np.zeros((n, height, width), np.uint8)
    dep = np.zeros((n, height, width), np.float32)
    nrm = np.zeros((n, height, width, 3), np.float32)
    pts = np.zeros((num_points, 3), np.float64)
    off = np.zeros(num_points + 1, np.uint32)
    tv = np.zeros(max(num_points * n, 1), np.uint32)
    npts = C.c_int(0)
    rc = _synth_lib().synth_reference_scene(C.byref(cfg), cams.ctypes.data, gray.ctypes.data, dep.ctypes.data,
                                            nrm.ctypes.data, pts.ctypes.data, off.ctypes.data, tv.ctypes.data,
                                            C.byref(npts))
    if rc != 0:
        raise RuntimeError("synth_reference_scene failed")
    m = npts.value
    cam_list = []
    for v in range(n):
        j, i = divmod(v, grid[0])
        c = cams[v]
        cam_list.append(Camera(f"synth_{j}_{i}.png", tuple(float(x) for x in c[:4]), c[4:13].reshape(3, 3).copy(),
                               c[13:16].copy(), width, height))
    views = np.array([np.concatenate([c.r.ravel(), c.t]) for c in cam_list], np.float64)
    model = SparseModel(views, np.ascontiguousarray(pts[:m]), off[: m + 1].copy(), tv[: off[m]].copy())
    return ReferenceScene(cam_list, gray, dep, nrm, model, tuple(boxes))
