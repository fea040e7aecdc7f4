"""The FP64 oracle of the proposal network (oracle/cnn_oracle.py), pinned by mathematics: its analytic parameter
gradients equal central finite differences of its own loss, and its bf16 rounding is round-to-nearest-even.  The GPU
kernels are then checked against this oracle (tests/test_gpu_proposal.py)."""
import numpy as np
import pytest

from oracle import cnn_oracle as O
from cumulus3d_b200 import proposal


def _params(rng):
    flat = []
    for ci, co in O.LAYERS:
        b = np.sqrt(6.0 / (9 * ci))
        flat.append(rng.uniform(-b, b, co * 9 * ci))
        flat.append(rng.uniform(-0.1, 0.1, co))
    return np.concatenate(flat)


def _batch(rng, b, h, w, dr=(25.0, 60.0)):
    x = rng.uniform(0, 1, (b, h, w, 48))
    x[..., 33:] = 0
    lab = np.zeros((b, h, w, 6))
    lab[..., 0] = rng.uniform(0, 1, (b, h, w))
    n = rng.normal(size=(b, h, w, 3))
    lab[..., 1:4] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    lab[..., 4] = rng.random((b, h, w)) < 0.8
    d = 1.0 / (1.0 / dr[1] + lab[..., 0] * (1.0 / dr[0] - 1.0 / dr[1]))
    lab[..., 5] = d * (1 + rng.normal(0, 0.01, (b, h, w)))
    return x, lab


def test_layer_table_matches_engine_header():
    assert O.LAYERS == proposal.LAYERS
    assert proposal.NUM_PARAMS == sum(co * 9 * ci + co for ci, co in O.LAYERS)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 3.140625, 1e-3], np.float64)
    bits = O.bf16_bits(v)
    assert bits[0] == 0x3F80
    assert bits[1] == 0x3F80  # tie -> even
    assert bits[2] == 0x3F82  # tie -> even (up)
    assert bits[3] == 0x3F80
    assert bits[4] == 0xC020
    np.testing.assert_array_equal(O.from_bf16_bits(bits), O.bf16_round(v))


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    flat = _params(rng)
    x, lab = _batch(rng, 1, 16, 16)
    a = O.forward(O.split(flat), x)
    loss, g_o = O.loss_and_grad(a["o"], lab, (25.0, 60.0))
    grad = O.backward(O.split(flat), a, g_o)
    assert np.isfinite(loss) and loss > 0
    # probe every layer: its first bias and weights on live input channels
    probes, o = [], 0
    for ci, co in O.LAYERS:
        nw = co * 9 * ci
        live = [i for i in range(o, o + nw) if (i - o) % ci < (33 if ci == 48 else ci)]
        probes += list(rng.choice(live, 2, replace=False)) + [o + nw, o + nw + co - 1]
        o += nw + co
    checked = 0
    for i in probes:
        e = 1e-5
        fp, fm = flat.copy(), flat.copy()
        fp[i] += e
        fm[i] -= e
        fd = (O.loss_of(fp, x, lab, (25.0, 60.0)) - O.loss_of(fm, x, lab, (25.0, 60.0))) / (2 * e)
        assert abs(grad[i] - fd) <= 1e-4 * abs(fd) + 1e-9, (i, grad[i], fd)
        checked += grad[i] != 0.0
    assert checked >= len(probes) // 2


def test_oracle_conv_grads_are_adjoint():
    """<conv(x, w), dy> = <x, dx> = <w, dw>: the data and weight gradients are the adjoints of the convolution."""
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 5, 7, 16))
    w = rng.normal(size=(8, 9, 16))
    dy = rng.normal(size=(2, 5, 7, 8))
    y = O.conv(x, w)
    dx, dw, db = O.conv_grads(x, w, dy)
    ip = (y * dy).sum()
    assert abs(ip - (x * dx).sum()) < 1e-9 * abs(ip) + 1e-9
    assert abs(ip - (w * dw).sum()) < 1e-9 * abs(ip) + 1e-9
    np.testing.assert_allclose(db, dy.reshape(-1, 8).sum(0))
