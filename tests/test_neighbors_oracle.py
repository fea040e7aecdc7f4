"""Neighbour views and depth ranges (crates/dense/src/neighbors.rs:44-186): the CPU oracle against the reference's own
known answers, against an independent pure-Python restatement (the direction-diverse path has no reference answer),
and the engine's host-side input validation (no GPU needed)."""
import ctypes as C
import math

import numpy as np
import pytest

from cumulus3d_b200 import _lib
from cumulus3d_b200.neighbors import NeighborParams, SparseModel
from oracle import oracle


def _down_view(c):
    """A camera at c looking straight down (rotation diag(1, -1, -1))."""
    r = np.diag([1.0, -1.0, -1.0])
    return r, np.array([-(r[0, 0] * c[0]), -(r[1, 1] * c[1]), -(r[2, 2] * c[2])])


def known_answer_model() -> SparseModel:
    """The scene of crates/dense/tests/host_parts.rs:62-84: views 10 m up at x = 0, 3 (large angle), 0.05 (angle
    below 1 degree) and -3; 5 points shared by views 0-1, 8 by 0-2, 3 by 0-3 and 1 by 1-3."""
    vs = [_down_view(c) for c in ([0, 0, 10], [3, 0, 10], [0.05, 0, 10], [-3, 0, 10])]
    pts, tracks = [], []
    for n, a, b in ((5, 0, 1), (8, 0, 2), (3, 0, 3), (1, 1, 3)):
        for k in range(n):
            pts.append([k * 0.1, 0.0, 0.0])
            tracks.append([a, b])
    return SparseModel.from_tracks([v[0] for v in vs], [v[1] for v in vs], np.array(pts), tracks)


def test_selection_and_depth_range_known_answers():
    m = known_answer_model()
    assert oracle.select_neighbors(m, NeighborParams(10, 1.0)).sources[0] == [1, 3]
    assert oracle.select_neighbors(m, NeighborParams(1, 1.0)).sources[0] == [1]
    assert oracle.select_neighbors(m, NeighborParams(10, 0.0)).sources[0] == [2, 1, 3]
    r = oracle.select_neighbors(m, NeighborParams(10, 1.0))
    assert r.sources[1] == [0, 3]
    lo, hi = r.depth_ranges[0]
    assert abs(lo - 7.5) < 1e-9 and abs(hi - 12.5) < 1e-9


def test_depth_range_of_known_answer():
    """depth_range_of over depths 1..100 gives (1.5, 125) (neighbors.rs:189-197): one view at the origin looking
    along +z sees points at z = 1..100, each shared with a second view."""
    r = np.eye(3)
    views = [(r, np.zeros(3)), (r, np.array([1.0, 0.0, 0.0]))]
    pts = np.array([[0.0, 0.0, float(z)] for z in range(1, 101)])
    m = SparseModel.from_tracks([v[0] for v in views], [v[1] for v in views], pts, [[0, 1]] * 100)
    lo, hi = oracle.select_neighbors(m, NeighborParams(2, 0.0)).depth_ranges[0]
    assert abs(lo - 1.5) < 1e-12 and abs(hi - 125.0) < 1e-12


def random_model(seed: int, nv: int = 9, npts: int = 400, max_track: int = 6) -> SparseModel:
    rng = np.random.default_rng(seed)
    rots, ts = [], []
    for _ in range(nv):
        c = rng.uniform([-20, -20, 25], [20, 20, 35])
        a = rng.normal(size=3) * 0.3
        k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        r = np.diag([1.0, -1.0, -1.0]) @ (np.eye(3) + k + k @ k / 2)
        u, _, vt = np.linalg.svd(r)
        r = u @ vt
        rots.append(r)
        ts.append(-r @ c)
    xyz = rng.uniform([-30, -30, -2], [30, 30, 6], size=(npts, 3))
    tracks = []
    for _ in range(npts):
        L = int(rng.integers(0, max_track + 1))
        t = list(rng.integers(0, nv - 1, size=L))  # the last view is never observed
        if L >= 3 and rng.random() < 0.1:
            t.append(t[0])  # a repeated view in a track counts as the reference counts it
        tracks.append([int(v) for v in t])
    return SparseModel.from_tracks(rots, ts, xyz, tracks)


def python_restatement(m: SparseModel, p: NeighborParams):
    """A second, independent restatement of neighbors.rs:47-186 in Python floats (math.acos / math.atan2 are the
    platform's, as the reference's f64 functions are)."""
    n = m.num_views
    R = [m.views[i, :9].reshape(3, 3) for i in range(n)]
    T = [m.views[i, 9:] for i in range(n)]
    cen = [[-(R[v][0][j] * T[v][0] + R[v][1][j] * T[v][1] + R[v][2][j] * T[v][2]) for j in range(3)] for v in range(n)]
    pairs = {}
    for i in range(len(m.track_offsets) - 1):
        x = [float(q) for q in m.xyz[i]]
        tr = [int(v) for v in m.track_views[m.track_offsets[i]:m.track_offsets[i + 1]]]
        for a_i in range(len(tr)):
            for b_i in range(a_i):
                a, b = tr[a_i], tr[b_i]
                if a == b:
                    continue
                u = [cen[a][k] - x[k] for k in range(3)]
                w = [cen[b][k] - x[k] for k in range(3)]
                nu = math.sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
                nw = math.sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2])
                ang = 0.0
                if not (nu == 0.0 or nw == 0.0):
                    c = (u[0] * w[0] + u[1] * w[1] + u[2] * w[2]) / (nu * nw)
                    c = min(max(c, -1.0), 1.0)
                    t = math.acos(c)
                    ang = min(t, math.pi - t)
                e = pairs.setdefault((min(a, b), max(a, b)), [0, []])
                e[0] += 1
                e[1].append(float(np.float32(ang)))

    def q75(v):
        v = sorted(v)
        pos = 0.75 * (len(v) - 1)
        lo = math.floor(pos)
        hi = min(lo + 1, len(v) - 1)
        return v[lo] + (v[hi] - v[lo]) * (pos - lo)

    def powi(a, b):
        r = 1.0
        while True:
            if b & 1:
                r *= a
            b //= 2
            if b == 0:
                break
            a *= a
        return r

    min_angle = p.min_triangulation_angle_deg * (math.pi / 180.0)
    out = []
    for r in range(n):
        cands = []
        for o in range(n):
            e = pairs.get((min(r, o), max(r, o)))
            if o == r or e is None:
                continue
            if min_angle > 0.0 and q75(e[1]) < min_angle:
                continue
            cands.append((e[0], o))
        cands.sort(key=lambda co: (-co[0], co[1]))
        if p.diversity_decay >= 1.0:
            out.append([o for _, o in cands[:p.num_views]])
            continue
        bins = max(p.direction_bins, 1)
        info = []
        for cnt, o in cands:
            d = [cen[o][k] - cen[r][k] for k in range(3)]
            b = [R[r][k][0] * d[0] + R[r][k][1] * d[1] + R[r][k][2] * d[2] for k in range(3)]
            lat = math.sqrt(b[0] * b[0] + b[1] * b[1])
            bn = bins if lat < 0.3 * abs(b[2]) else min(int((math.atan2(b[1], b[0]) + math.pi) / (2.0 * math.pi) * bins),
                                                        bins - 1)
            info.append((o, float(cnt), bn))
        used = [0] * (bins + 1)
        taken = [False] * len(info)
        sel = []
        while len(sel) < p.num_views:
            best = None
            for i, (_, sc, bn) in enumerate(info):
                if taken[i]:
                    continue
                s = sc * powi(p.diversity_decay, used[bn])
                if best is None or s > best[0]:
                    best = (s, i)
            if best is None:
                break
            taken[best[1]] = True
            used[info[best[1]][2]] += 1
            sel.append(info[best[1]][0])
        out.append(sel)
    return out


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("params", [NeighborParams(4, 1.0), NeighborParams(10, 0.0), NeighborParams(3, 5.0),
                                    NeighborParams(4, 1.0, 8, 0.5), NeighborParams(6, 0.0, 4, 0.25)])
def test_oracle_equals_independent_restatement(seed, params):
    m = random_model(seed)
    assert oracle.select_neighbors(m, params).sources == python_restatement(m, params)


def test_invalid_tracks_are_rejected_before_any_device_work():
    m = known_answer_model()
    bad = SparseModel(m.views, m.xyz, m.track_offsets, m.track_views.copy())
    bad.track_views[3] = 7  # view index out of range
    lib = _lib.engine()
    from cumulus3d_b200 import neighbors
    with pytest.raises(_lib.PsError) as e:
        neighbors.call(lib.ps_select_neighbors, bad, NeighborParams(), False, 0)
    assert e.value.code == _lib.PS_EINVAL
    with pytest.raises(_lib.PsError) as e:
        neighbors.call(lib.ps_select_neighbors, m, NeighborParams(0, 1.0), False, 0)
    assert e.value.code == _lib.PS_EINVAL


def test_sparse_model_of_views_of_different_sizes():
    """Tracks from depth maps of different sizes (one map per view, not a stacked array)."""
    from cumulus3d_b200 import scenes
    cams = scenes.formation(64, 48, 1, prefix="a") + scenes.formation(96, 72, 1, prefix="b", y0=1.0)
    depth = [np.full((c.height, c.width), 30.0, np.float32) for c in cams]
    m = scenes.sparse_model(cams, depth, 200, seed=1, rel_tol=0.5)
    assert m.num_views == len(cams) and len(m.track_offsets) == m.xyz.shape[0] + 1
    assert int(m.track_offsets[-1]) == m.track_views.size and m.track_views.max() < len(cams)
    r = oracle.select_neighbors(m, NeighborParams(2, 0.0))
    assert len(r.sources) == len(cams)
