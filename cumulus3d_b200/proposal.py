"""Learned proposal for the PatchStereo engine (no reference counterpart).

A BF16 encoder-decoder (``ps_net_*`` in include/patchstereo.h, kernels in csrc/ps_cnn.cu) predicts an initial plane and
a confidence per pixel from the reference image and a 32-plane NCC sweep volume (``ps_sweep_volume``).  A photometric
run that starts with ``random_init = PS_INIT_PROPOSAL`` takes the proposed plane wherever the confidence reached the
threshold and the ordinary seeded random draw everywhere else, so plain PatchStereo initialisation is the per-pixel
fallback, and the PatchStereo iterations that follow decide every pixel's final plane.

Training data are the engine's own outputs: seeded synthetic terrains seen through the 1920×1080 camera formation of
the aerial workloads, cut into 256×256 reference crops (a crop is the same camera with a shifted principal point)
whose sources are windows of the neighbouring cameras covering the crop's footprint over the whole depth range.  The
label of a crop is the plane field of a 6-iteration plain photometric run on it, valid where its matching cost is
below ``LABEL_MAX_COST``.  Training runs on the GPU through ``ps_net_train_step`` (forward, loss, backward and AdamW
in the project's own kernels).

PyTorch only provides device buffers here (the network input and labels of the training set); every kernel is the
engine's.
"""
from __future__ import annotations

import ctypes as C
import math
import pathlib
import time
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib, scenes
from .patchstereo import KernelInput, PatchMatchBackend, RunParams, ViewState

# (cin, cout) of the 12 3×3 convolutions in parameter order (e0a e0b e1a e1b e2a e2b e3a e3b d2 d1 d0 head).
LAYERS: Tuple[Tuple[int, int], ...] = ((48, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (96, 128),
                                       (128, 128), (224, 96), (160, 64), (96, 32), (32, 8))
LAYER_NAMES = ("e0a", "e0b", "e1a", "e1b", "e2a", "e2b", "e3a", "e3b", "d2", "d1", "d0", "head")
NUM_PARAMS = sum(co * 9 * ci + co for ci, co in LAYERS)
WEIGHTS_DIR = pathlib.Path(__file__).resolve().parent / "weights"
DEFAULT_WEIGHTS = WEIGHTS_DIR / "proposal_aerial.npz"
LABEL_MAX_COST = 0.6
CONF_THRESHOLD = 0.15


def split_params(flat: np.ndarray):
    """Flat parameter vector -> [(W (cout, 9, cin), b (cout,))] per layer."""
    out, o = [], 0
    for ci, co in LAYERS:
        w = flat[o:o + co * 9 * ci].reshape(co, 9, ci)
        o += co * 9 * ci
        b = flat[o:o + co]
        o += co
        out.append((w, b))
    assert o == flat.size
    return out


class ProposalNet:
    """Owner of one ``ps_net`` (parameters, AdamW state and workspace on one GPU)."""

    def __init__(self, device: int = 0, seed: int = 1, weights: Optional[pathlib.Path] = None):
        self.lib = _lib.engine()
        self.device = device
        h = C.c_void_p()
        rc = self.lib.ps_net_create(device, seed, C.byref(h))
        if rc != _lib.PS_OK:
            raise _lib.PsError(rc, "ps_net_create failed")
        self.h = h
        if self.num_params != NUM_PARAMS:
            raise RuntimeError(f"network layout mismatch: {self.num_params} != {NUM_PARAMS} parameters")
        if weights is not None:
            self.load(weights)

    def _check(self, rc: int):
        if rc != _lib.PS_OK:
            raise _lib.PsError(rc, self.lib.ps_net_last_error(self.h).decode())

    @property
    def num_params(self) -> int:
        return int(self.lib.ps_net_num_params(self.h))

    @property
    def step(self) -> int:
        return int(self.lib.ps_net_step(self.h))

    def get_params(self) -> np.ndarray:
        out = np.empty(self.num_params, np.float32)
        self._check(self.lib.ps_net_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_params(self, flat: np.ndarray) -> None:
        a = np.ascontiguousarray(flat, np.float32)
        assert a.size == self.num_params
        self._check(self.lib.ps_net_set_params(self.h, a.ctypes.data_as(C.POINTER(C.c_float))))

    def save(self, path: pathlib.Path, meta: Optional[dict] = None) -> None:
        path = pathlib.Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, params=self.get_params(), layers=np.array(LAYERS, np.int32),
                            meta=np.array(repr(meta or {})))

    def load(self, path: pathlib.Path) -> None:
        z = np.load(pathlib.Path(path))
        if tuple(map(tuple, z["layers"].tolist())) != LAYERS:
            raise RuntimeError(f"{path}: layer table differs from this network")
        self.set_params(z["params"])

    def forward(self, x, out, stream: int = 0) -> None:
        """x: CUDA tensor (B, H, W, 48) of bf16 bits (int16/uint16/bfloat16); out: CUDA float32 (B, H, W, 8)."""
        b, hh, ww, c = x.shape
        assert c == _lib.PS_NET_CH_IN and tuple(out.shape) == (b, hh, ww, _lib.PS_NET_CH_OUT)
        self._check(self.lib.ps_net_forward(self.h, C.c_void_p(x.data_ptr()), b, hh, ww, C.c_void_p(out.data_ptr()),
                                            C.c_void_p(stream) if stream else None))

    def train_step(self, x, labels, depth_range: Tuple[float, float], lr: float, weight_decay: float = 1e-4,
                   grads: bool = False):
        """One AdamW step (lr = 0: loss and gradients only).  Returns loss, or (loss, gradient vector)."""
        b, hh, ww, _ = x.shape
        loss = C.c_float()
        g = np.empty(self.num_params, np.float32) if grads else None
        self._check(self.lib.ps_net_train_step(
            self.h, C.c_void_p(x.data_ptr()), C.c_void_p(labels.data_ptr()), b, hh, ww, depth_range[0],
            depth_range[1], lr, weight_decay, C.byref(loss), g.ctypes.data_as(C.POINTER(C.c_float)) if grads else None))
        return (loss.value, g) if grads else loss.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ps_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_conv_path(path: str) -> None:
    """'auto' (default: tcgen05 for cout >= 64, mma.sync otherwise), 'mma' (mma.sync only) or 'tcgen05' (tcgen05 for
    every cout in {32, 64, 96, 128})."""
    rc = _lib.engine().ps_net_set_conv_path({"auto": 0, "mma": 1, "tcgen05": 2}[path])
    if rc != _lib.PS_OK:
        raise _lib.PsError(rc, "ps_net_set_conv_path failed")


def conv_timeouts(device: int = 0, reset: bool = False) -> int:
    """Expired bounded waits of the tcgen05 convolution on `device` (0 when every result is valid)."""
    c = C.c_uint32()
    rc = _lib.engine().ps_net_conv_timeouts(device, C.byref(c), int(reset))
    if rc != _lib.PS_OK:
        raise _lib.PsError(rc, "ps_net_conv_timeouts failed")
    return int(c.value)


def conv_check(x: np.ndarray, w: np.ndarray, dy: np.ndarray, device: int = 0):
    """One convolution forward / data gradient / weight gradient through the network's kernels (host buffers).
    x (B, H, W, cin) and dy (B, H, W, cout) uint16 bf16 bits; w (cout, 9, cin) f32."""
    b, hh, ww, ci = x.shape
    co = w.shape[0]
    x = np.ascontiguousarray(x, np.uint16)
    dy = np.ascontiguousarray(dy, np.uint16)
    w = np.ascontiguousarray(w, np.float32)
    y = np.empty((b, hh, ww, co), np.float32)
    dx = np.empty((b, hh, ww, ci), np.float32)
    dw = np.empty_like(w)
    rc = _lib.engine().ps_net_conv_check(device, x.ctypes.data, w.ctypes.data, dy.ctypes.data, b, hh, ww, ci, co,
                                         y.ctypes.data, dx.ctypes.data, dw.ctypes.data)
    if rc != _lib.PS_OK:
        raise _lib.PsError(rc, "ps_net_conv_check failed")
    return y, dx, dw


# ---------------------------------------------------------------------------------------------- labels
def make_labels(depth: np.ndarray, normal: np.ndarray, valid: np.ndarray, depth_range: Tuple[float, float],
                out: Optional[np.ndarray] = None) -> np.ndarray:
    """(H, W, 6) f32: t* = (1/d - 1/dmax) / (1/dmin - 1/dmax), normal xyz, valid, d."""
    dmin, dmax = depth_range
    h, w = depth.shape
    lab = out if out is not None else np.zeros((h, w, 6), np.float32)
    ok = valid & (depth > 0)
    inv = np.where(ok, 1.0 / np.maximum(depth, 1e-6), 0.0)
    lab[..., 0] = np.clip((inv - 1.0 / dmax) / (1.0 / dmin - 1.0 / dmax), 0.0, 1.0)
    lab[..., 1:4] = normal
    lab[..., 4] = ok
    lab[..., 5] = depth
    lab[~ok] = 0.0
    return lab


# ---------------------------------------------------------------------------------------------- training scenes
@dataclass
class CropScene:
    """One training sample: a reference crop and source windows of the same terrain (their cameras and images)."""
    cams: List[scenes.Camera]
    images: List[np.ndarray]
    seed: int


def _project(cam: scenes.Camera, pts: np.ndarray) -> np.ndarray:
    pc = pts @ cam.r.T + cam.t
    fx, fy, cx, cy = cam.k
    return np.stack([fx * pc[:, 0] / pc[:, 2] + cx, fy * pc[:, 1] / pc[:, 2] + cy], axis=1)


def _shifted(cam: scenes.Camera, x0: int, y0: int, w: int, h: int, name: str) -> scenes.Camera:
    fx, fy, cx, cy = cam.k
    return scenes.Camera(name, (fx, fy, cx - x0, cy - y0), cam.r, cam.t, w, h)


def crop_scene(seed: int, crop: int = 256, depth_range=(25.0, 60.0), sources: int = 4, window_radius: int = 6,
               full=(1920, 1080)) -> CropScene:
    """A reference crop of the aerial formation (same intrinsics as the 1920×1080 workloads) and windows of its
    `sources` nearest cameras covering the crop's footprint between the depth bounds (+ the window radius)."""
    rng = np.random.default_rng(seed)
    fw, fh = full
    cams = scenes.formation(fw, fh, 3, prefix=f"tr{seed}")
    ref_i = int(rng.integers(0, len(cams)))  # any camera: end stations see other source geometries than the middle
    near = scenes.nearest_sources(cams, sources)[ref_i]
    ext = scenes._extent(cams)
    x0 = int(rng.integers(0, (fw - crop) // 8 + 1)) * 8
    y0 = int(rng.integers(0, (fh - crop) // 8 + 1)) * 8
    ref = _shifted(cams[ref_i], x0, y0, crop, crop, f"tr{seed}_ref")
    fx, fy, cx, cy = ref.k
    us = np.array([0, crop - 1, 0, crop - 1, crop / 2, 0, crop - 1, crop / 2], np.float64)
    vs = np.array([0, 0, crop - 1, crop - 1, crop / 2, crop / 2, crop / 2, 0], np.float64)
    rays = np.stack([(us - cx) / fx, (vs - cy) / fy, np.ones_like(us)], axis=1)
    pts = []
    for d in np.linspace(depth_range[0], depth_range[1], 4):
        pc = rays * d  # camera coordinates, z = depth
        pts.append((pc - ref.t) @ ref.r)  # world = Rᵀ (pc - t)
    pts = np.concatenate(pts)
    out_cams, m = [ref], window_radius + 8
    for j in near:
        uv = _project(cams[j], pts)
        sx0 = max(0, int(math.floor((uv[:, 0].min() - m) / 8)) * 8)
        sy0 = max(0, int(math.floor((uv[:, 1].min() - m) / 8)) * 8)
        sx1 = min(fw, int(math.ceil((uv[:, 0].max() + m) / 8)) * 8)
        sy1 = min(fh, int(math.ceil((uv[:, 1].max() + m) / 8)) * 8)
        if sx1 - sx0 < 16 or sy1 - sy0 < 16:
            sx0, sy0, sx1, sy1 = 0, 0, fw, fh
        out_cams.append(_shifted(cams[j], sx0, sy0, sx1 - sx0, sy1 - sy0, f"tr{seed}_s{j}"))
    images = []
    for c in out_cams:
        img, _, _ = scenes.render([c], seed, with_gt=False, extent=ext)
        images.append(img[0])
    return CropScene(out_cams, images, seed)


def crop_input(group: Sequence[CropScene], depth_range=(25.0, 60.0), window_radius: int = 6) -> Tuple[KernelInput, List[int]]:
    """One KernelInput over several crop scenes; returns it and the indices of the reference views."""
    cams, images, sources, refs = [], [], [], []
    for sc in group:
        base = len(cams)
        refs.append(base)
        cams += sc.cams
        images += sc.images
        sources.append([base + j for j in range(1, len(sc.cams))])
        for j in range(1, len(sc.cams)):
            sources.append([base])  # sources need a source of their own to form a valid view; they are never run
    inp = scenes.kernel_input(cams, images, sources, depth_range, window_radius=window_radius, window_step=1)
    return inp, refs


@dataclass
class TrainingSet:
    x: "object"       # torch CUDA int16 (N, H, W, 48) bf16 bits
    labels: "object"  # torch CUDA float32 (N, H, W, 6)
    depth_range: Tuple[float, float]
    valid_fraction: float
    seconds: dict


def make_training_set(n_scenes: int = 300, seed: int = 1000, crop: int = 256, depth_range=(25.0, 60.0),
                      label_iters: int = 6, group: int = 30, device: int = 0, log=print) -> TrainingSet:
    """Renders `n_scenes` seeded crop scenes, labels them with the engine's plain photometric PatchStereo
    (`label_iters` iterations, random init) and sweeps their network inputs, all kept on the GPU."""
    import torch

    dev = torch.device("cuda", device)
    xs = torch.empty((n_scenes, crop, crop, _lib.PS_NET_CH_IN), dtype=torch.int16, device=dev)
    torch.cuda.synchronize(dev)  # the session stream that fills xs does not wait for torch's stream
    labs = np.zeros((n_scenes, crop, crop, 6), np.float32)
    t_render = t_label = 0.0
    be = PatchMatchBackend(device, math="parity")
    done = 0
    for g0 in range(0, n_scenes, group):
        t0 = time.time()
        grp = [crop_scene(seed + i, crop, depth_range) for i in range(g0, min(n_scenes, g0 + group))]
        inp, refs = crop_input(grp, depth_range)
        t_render += time.time() - t0
        t0 = time.time()
        states = [ViewState.new(crop, crop) for _ in refs]
        with be.begin(inp) as s:
            s.run(refs, states, RunParams(0, False, True, label_iters, 1))
            for i, v in enumerate(refs):
                s.sweep_volume(0, v, xs[g0 + i].data_ptr(), crop)
            s.synchronize()
        for i, st in enumerate(states):
            make_labels(st.depth, st.normal, st.cost < LABEL_MAX_COST, depth_range, labs[g0 + i])
        t_label += time.time() - t0
        done += len(grp)
        if log:
            log(f"training set: {done}/{n_scenes} scenes (render {t_render:.1f}s, label+sweep {t_label:.1f}s)")
    be.close()
    lab_t = torch.from_numpy(labs).to(dev)
    return TrainingSet(xs, lab_t, depth_range, float(labs[..., 4].mean()),
                       {"render": t_render, "label_sweep": t_label})


def train(net: ProposalNet, data: TrainingSet, steps: int = 1500, batch: int = 8, lr: float = 1e-3,
          weight_decay: float = 1e-4, seed: int = 0, log=print, log_every: int = 100) -> List[float]:
    """AdamW on random batches of the training set; returns the per-step losses."""
    import torch

    rng = np.random.default_rng(seed)
    n = data.x.shape[0]
    losses = []
    t0 = time.time()
    for it in range(steps):
        idx = torch.from_numpy(rng.choice(n, size=min(batch, n), replace=False)).to(data.x.device)
        xb = data.x.index_select(0, idx).contiguous()
        lb = data.labels.index_select(0, idx).contiguous()
        torch.cuda.synchronize(data.x.device)
        losses.append(net.train_step(xb, lb, data.depth_range, lr, weight_decay))
        if log and (it % log_every == 0 or it == steps - 1):
            log(f"step {it}: loss {losses[-1]:.4f} ({time.time() - t0:.1f}s)")
    return losses


# ---------------------------------------------------------------------------------------------- evaluation
def agreement(depth: np.ndarray, ref: np.ndarray, mask: Optional[np.ndarray] = None, tol: float = 0.01) -> float:
    """Fraction of pixels (ref > 0, and `mask`) whose depth is within `tol` relative of `ref`."""
    m = ref > 0
    if mask is not None:
        m &= mask
    if not m.any():
        return float("nan")
    return float((np.abs(depth[m] - ref[m]) <= tol * ref[m]).mean())


def evaluate_gain(net: ProposalNet, n_scenes: int = 6, seed: int = 90000, crop: int = 256, iters: int = 2,
                  plain_iters: int = 6, depth_range=(25.0, 60.0), device: int = 0,
                  threshold: float = CONF_THRESHOLD) -> dict:
    """Held-out crop scenes: agreement (within 1 % depth) with the plain `plain_iters`-iteration result, on pixels
    where that result's cost is below LABEL_MAX_COST, of (a) `iters` iterations from random init and (b) `iters`
    iterations from the learned proposal (random init where the confidence is below `threshold`)."""
    grp = [crop_scene(seed + i, crop, depth_range) for i in range(n_scenes)]
    inp, refs = crop_input(grp, depth_range)
    be = PatchMatchBackend(device, math="parity")
    plain = [ViewState.new(crop, crop) for _ in refs]
    rnd = [ViewState.new(crop, crop) for _ in refs]
    lrn = [ViewState.new(crop, crop) for _ in refs]
    with be.begin(inp) as s:
        s.run(refs, plain, RunParams(0, False, True, plain_iters, 1))
        s.run(refs, rnd, RunParams(0, False, True, iters, 1))
        proposed = s.propose(net, 0, refs, threshold)
        s.run(refs, lrn, RunParams(0, False, _lib.PS_INIT_PROPOSAL, iters, 1))
    be.close()
    a_r = [agreement(r.depth, p.depth, p.cost < LABEL_MAX_COST) for r, p in zip(rnd, plain)]
    a_l = [agreement(l.depth, p.depth, p.cost < LABEL_MAX_COST) for l, p in zip(lrn, plain)]
    return {"random": float(np.nanmean(a_r)), "learned": float(np.nanmean(a_l)),
            "proposed_fraction": proposed / float(len(refs) * crop * crop), "iters": iters,
            "plain_iters": plain_iters, "scenes": n_scenes, "threshold": threshold}
