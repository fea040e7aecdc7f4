"""The footprint bound behind the staged source boxes of the half step (PS_TUNE_STAGED).

A warp stages the union of its lanes' source footprints into a shared-memory box and every tap reads its 2×2 texels
from there, so the box must contain every texel a tap reads, and the kernel's box address (a float added with
rounding toward -infinity, then its bits) must equal floor(u) minus the box origin.  The kernel's per-lane rule is
restated in the oracle (oracle_box_footprint_check); this test runs it over plane-induced homographies of realistic
camera pairs and over adversarial matrices: every window the rule accepts must have no tap outside its range, and
the rule must accept the ordinary windows (otherwise the staged path would never run).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle


def _check(H, x, y, wr, ws):
    h = (C.c_float * 9)(*[float(v) for v in H])
    rng = (C.c_int * 4)()
    return oracle.lib().oracle_box_footprint_check(h, int(x), int(y), int(wr), int(ws), rng), tuple(rng)


def _rot(rng, max_deg):
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    a = np.deg2rad(rng.uniform(-max_deg, max_deg))
    k = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    return np.eye(3) + np.sin(a) * k + (1 - np.cos(a)) * k @ k


def _plane_homography(rng, w, h):
    """H = K_j (R + t nᵀ / δ) K⁻¹ for a random pixel plane seen from a displaced, rotated source camera."""
    f = rng.uniform(0.6, 1.4) * w
    K = np.array([[f, 0, w / 2], [0, f, h / 2], [0, 0, 1.0]])
    R = _rot(rng, 12.0)
    t = rng.normal(size=3) * rng.uniform(0.5, 15.0)
    n = rng.normal(size=3)
    n[2] = -abs(n[2]) - 0.3
    n /= np.linalg.norm(n)
    d = rng.uniform(15.0, 90.0)
    Hm = K @ (R - np.outer(t, n) / (-d)) @ np.linalg.inv(K)
    return (Hm / Hm[2, 2]).astype(np.float32).ravel()


@pytest.mark.parametrize("wr,ws", [(3, 1), (5, 1), (5, 2), (6, 1), (20, 1)])
def test_realistic_windows_stay_inside_their_box(wr, ws):
    rng = np.random.default_rng(100 + wr * 3 + ws)
    accepted = 0
    n = 3000
    for _ in range(n):
        w, h = (3840, 2160) if rng.random() < 0.3 else (1920, 1080)
        H = _plane_homography(rng, w, h)
        bad, _ = _check(H, rng.integers(0, w), rng.integers(0, h), wr, ws)
        assert bad <= 0, (bad, H.tolist())
        accepted += bad == 0
    assert accepted > 0.8 * n, accepted


def test_adversarial_matrices():
    """Heavy-tailed entries, near-degenerate depths, huge translations, NaN and infinity: whatever the rule accepts
    must still hold, and non-finite matrices are rejected."""
    rng = np.random.default_rng(7)
    accepted = 0
    for k in range(6000):
        H = (rng.standard_cauchy(9) * 10.0 ** rng.uniform(-3, 4, 9)).astype(np.float32)
        if k % 3 == 0:
            H[6:8] = (rng.normal(size=2) * 1e-3).astype(np.float32)
            H[8] = np.float32(rng.uniform(1e-7, 2.0))
        bad, _ = _check(H, rng.integers(0, 4096), rng.integers(0, 4096), 6, 1)
        assert bad <= 0, (bad, H.tolist())
        accepted += bad == 0
    assert accepted > 0
    for v in (np.nan, np.inf, -np.inf):
        for i in range(9):
            H = np.eye(3, dtype=np.float32).ravel()
            H[i] = v
            assert _check(H, 100, 100, 6, 1)[0] == -1


def test_box_of_identity_is_tight():
    """A unit homography (source = reference) gives the window itself plus one texel on the high side."""
    bad, (lx, hx, ly, hy) = _check(np.eye(3, dtype=np.float32).ravel(), 200, 100, 6, 1)
    assert bad == 0
    assert (lx, hx, ly, hy) == (200 - 6 - 1, 200 + 6 + 1, 100 - 6 - 1, 100 + 6 + 1)


def _place(g0, g1, size, align):
    """The kernel's box origin for a request [g0, g1] (inclusive) in a box of `size` texels: centred, and for x
    rounded to ≡ 2 (mod 4) (16-byte chunks of the bordered plane rows)."""
    lo = g1 - (size - 1)
    o = (lo + g0) >> 1
    if align:
        o -= (o - 2) & 3
        if o < lo:
            o += 4
    return o


def _box_dims():
    import pathlib
    import re
    hdr = (pathlib.Path(__file__).resolve().parent.parent / "cumulus3d_b200" / "csrc" / "ps_types.h").read_text()
    return (int(re.search(r"#define PS_BOX_P (\d+)", hdr).group(1)), int(re.search(r"#define PS_BOX_H (\d+)", hdr).group(1)))


def test_box_placement_contains_every_admissible_request():
    """Every request the kernel stages (at most PS_BOX_P - 3 wide, PS_BOX_H tall) lies inside the placed box, and the
    x origin keeps the 16-byte chunk alignment; the pitch is a whole number of 16-byte chunks."""
    bp, bh = _box_dims()
    assert bp % 4 == 0
    for g0 in range(-70, 70):
        for width in range(1, bp - 2):
            g1 = g0 + width - 1
            o = _place(g0, g1, bp, True)
            assert (o - 2) % 4 == 0 and o <= g0 and g1 <= o + bp - 1, (g0, g1, o)
        for height in range(1, bh + 1):
            g1 = g0 + height - 1
            o = _place(g0, g1, bh, False)
            assert o <= g0 and g1 <= o + bh - 1, (g0, g1, o)
