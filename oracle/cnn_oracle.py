"""FP64 CPU oracle of the learned-proposal network.  TEST INFRASTRUCTURE ONLY (tests/ use it as the checker of the
network kernels; the engine never imports it).

It restates, in numpy float64, the forward pass, the loss and the backward pass that csrc/ps_cnn.cu runs on the GPU:
3×3 "same" convolutions as im2col products (tap = 3·(dy+1) + (dx+1), weights [cout][9][cin]), ReLU, 2×2 average
pooling, nearest 2× upsampling, channel concatenation, the loss of ps_net_train_step and its gradient, and the
parameter gradients.  The network has no reference counterpart, so there is nothing to pin against other than
mathematics: tests check this oracle's gradients against central finite differences, then the GPU against this oracle.

With ``bf16=True`` the oracle rounds to bf16 exactly where the GPU stores bf16 (input, weights, every activation and
activation gradient), so GPU-vs-oracle differences come only from FP32 accumulation order.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

LAYERS = ((48, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (96, 128), (128, 128), (224, 96), (160, 64),
          (96, 32), (32, 8))


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round to the nearest bf16 (ties to even) via float32 bits; returns float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(a: np.ndarray) -> np.ndarray:
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def split(flat: np.ndarray) -> List[Tuple[np.ndarray, np.ndarray]]:
    out, o = [], 0
    for ci, co in LAYERS:
        w = np.asarray(flat[o:o + co * 9 * ci], np.float64).reshape(co, 9, ci)
        o += co * 9 * ci
        out.append((w, np.asarray(flat[o:o + co], np.float64)))
        o += co
    return out


def im2col(x: np.ndarray) -> np.ndarray:
    """(B, H, W, C) -> (B, H, W, 9, C) of the 3×3 neighbourhood (zero outside), tap = 3·(dy+1) + (dx+1)."""
    b, h, w, c = x.shape
    xp = np.zeros((b, h + 2, w + 2, c), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = np.empty((b, h, w, 9, c), x.dtype)
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        cols[:, :, :, t] = xp[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w]
    return cols


def col2im(cols: np.ndarray) -> np.ndarray:
    b, h, w, _, c = cols.shape
    xp = np.zeros((b, h + 2, w + 2, c), cols.dtype)
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        xp[:, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w] += cols[:, :, :, t]
    return xp[:, 1:-1, 1:-1]


def conv(x: np.ndarray, w: np.ndarray, b=None) -> np.ndarray:
    bb, h, ww, c = x.shape
    co = w.shape[0]
    y = im2col(x).reshape(-1, 9 * c) @ w.reshape(co, 9 * c).T
    if b is not None:
        y = y + b
    return y.reshape(bb, h, ww, co)


def conv_grads(x: np.ndarray, w: np.ndarray, dy: np.ndarray):
    """(dx, dw, db) of y = conv(x, w) + b."""
    bb, h, ww, c = x.shape
    co = w.shape[0]
    cols = im2col(x).reshape(-1, 9 * c)
    g = dy.reshape(-1, co)
    dw = (g.T @ cols).reshape(co, 9, c)
    dx = col2im((g @ w.reshape(co, 9 * c)).reshape(bb, h, ww, 9, c))
    return dx, dw, g.sum(axis=0)


def pool(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 1::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 1::2])


def pool_bwd(dy):
    return 0.25 * np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2)


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_bwd(dy):
    return dy[:, 0::2, 0::2] + dy[:, 1::2, 0::2] + dy[:, 0::2, 1::2] + dy[:, 1::2, 1::2]


def forward(params, x: np.ndarray, bf16: bool = False) -> Dict[str, np.ndarray]:
    """Forward pass; returns every activation (keys as in csrc/ps_cnn.cu) and the head output 'o'."""
    r = bf16_round if bf16 else (lambda a: a)
    P = [(r(w), b) for w, b in params]
    a: Dict[str, np.ndarray] = {"x": r(x)}

    def cr(name, inp, li, relu=True):
        y = conv(inp, *P[li])
        a[name] = r(np.maximum(y, 0.0)) if relu else y
        return a[name]

    cr("a0", a["x"], 0)
    cr("s0", a["a0"], 1)
    a["p1"] = r(pool(a["s0"]))
    cr("a1", a["p1"], 2)
    cr("s1", a["a1"], 3)
    a["p2"] = r(pool(a["s1"]))
    cr("a2", a["p2"], 4)
    cr("s2", a["a2"], 5)
    a["p3"] = r(pool(a["s2"]))
    cr("a3", a["p3"], 6)
    cr("b3", a["a3"], 7)
    a["c2"] = np.concatenate([up(a["b3"]), a["s2"]], axis=-1)
    cr("d2", a["c2"], 8)
    a["c1"] = np.concatenate([up(a["d2"]), a["s1"]], axis=-1)
    cr("d1", a["c1"], 9)
    a["c0"] = np.concatenate([up(a["d1"]), a["s0"]], axis=-1)
    cr("d0", a["c0"], 10)
    a["o"] = conv(a["d0"], *P[11])
    if bf16:
        a["o"] = a["o"].astype(np.float32).astype(np.float64)
    return a


def sigmoid(v):
    return 1.0 / (1.0 + np.exp(-v))


def loss_and_grad(o: np.ndarray, lab: np.ndarray, depth_range: Tuple[float, float]):
    """Mean loss over valid pixels and dL/do (same formulas as the GPU loss kernel)."""
    dmin, dmax = depth_range
    inv_near, inv_far = 1.0 / dmin, 1.0 / dmax
    valid = lab[..., 4] > 0.5
    n = max(int(valid.sum()), 1) if valid.any() else 0
    g = np.zeros_like(o)
    if n == 0:
        return 0.0, g
    t = sigmoid(o[..., 0])
    dt = t - lab[..., 0]
    loss = np.abs(dt)
    g[..., 0] = np.sign(dt) * t * (1 - t)
    nv = o[..., 1:4]
    ln = np.sqrt((nv ** 2).sum(-1)) + 1e-6
    c = (nv * lab[..., 1:4]).sum(-1) / ln
    loss = loss + 1 - c
    g[..., 1:4] = -(lab[..., 1:4] / ln[..., None] - c[..., None] * nv / (ln ** 2)[..., None])
    inv = inv_far + t * (inv_near - inv_far)
    d = 1.0 / np.maximum(inv, 1e-9)
    target = (np.abs(d - lab[..., 5]) < 0.01 * lab[..., 5]).astype(np.float64)
    cf = sigmoid(o[..., 4])
    loss = loss - 0.5 * (target * np.log(np.maximum(cf, 1e-7)) + (1 - target) * np.log(np.maximum(1 - cf, 1e-7)))
    g[..., 4] = 0.5 * (cf - target)
    g[~valid] = 0.0
    return float(loss[valid].sum() / n), g / n


def backward(params, a: Dict[str, np.ndarray], g_o: np.ndarray, bf16: bool = False) -> np.ndarray:
    """Parameter gradients (flat, parameter order) of the forward pass `a` for dL/do = g_o."""
    r = bf16_round if bf16 else (lambda v: v)
    P = [(r(w), b) for w, b in params]
    grads: List[Tuple[np.ndarray, np.ndarray]] = [None] * len(P)  # type: ignore

    def cb(li, dy, x, need_dx=True):
        dx, dw, db = conv_grads(x, P[li][0], dy)
        grads[li] = (dw, db)
        return r(dx) if need_dx else None

    def relu_mask(dy, y):
        return np.where(y > 0, dy, 0.0)

    g = cb(11, r(g_o), a["d0"])
    g = cb(10, relu_mask(g, a["d0"]), a["c0"])  # g_c0
    g_d1, g_s0 = r(up_bwd(g[..., :64])), g[..., 64:]
    g = cb(9, relu_mask(g_d1, a["d1"]), a["c1"])
    g_d2, g_s1 = r(up_bwd(g[..., :96])), g[..., 96:]
    g = cb(8, relu_mask(g_d2, a["d2"]), a["c2"])
    g_b3, g_s2 = r(up_bwd(g[..., :128])), g[..., 128:]
    g = cb(7, relu_mask(g_b3, a["b3"]), a["a3"])
    g = cb(6, relu_mask(g, a["a3"]), a["p3"])
    g_s2 = r(g_s2 + pool_bwd(g))
    g = cb(5, relu_mask(g_s2, a["s2"]), a["a2"])
    g = cb(4, relu_mask(g, a["a2"]), a["p2"])
    g_s1 = r(g_s1 + pool_bwd(g))
    g = cb(3, relu_mask(g_s1, a["s1"]), a["a1"])
    g = cb(2, relu_mask(g, a["a1"]), a["p1"])
    g_s0 = r(g_s0 + pool_bwd(g))
    g = cb(1, relu_mask(g_s0, a["s0"]), a["a0"])
    cb(0, relu_mask(g, a["a0"]), a["x"], need_dx=False)
    return np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads])


def loss_of(flat: np.ndarray, x: np.ndarray, lab: np.ndarray, depth_range) -> float:
    a = forward(split(flat), x)
    return loss_and_grad(a["o"], lab, depth_range)[0]
