"""Score fusion restated on the CPU (fuse_scored, crates/dense/src/fusion_score.rs:196-435), pinned by the
reference's own tests of that file (fuses_synthetic_scene_accurately, mark_used_reduces_duplicates,
point_count_monotone_in_tau, free_space_violations_are_rejected, deterministic_across_threads) on this package's
synthetic scene, by an independent pure-Python restatement of the per-pixel score, and by a check that the
reference's claim rounds choose what greedy selection in priority order chooses (the rule the restatement uses)."""
import math

import numpy as np
import pytest

from cumulus3d_b200 import fusion, scenes
from oracle import oracle


@pytest.fixture(scope="module")
def scene():
    wl = scenes.workload_small(160, 120, views=6, window_radius=3, seed=3, positions=2)
    src = [list(kv.sources) for kv in wl.input.views]
    return wl, fusion.FusionCams(wl.cams, src)


def _run(wl, fc, depths=None, costs=None, threads=None, **kw):
    """The reference tests' FusionInput::plain (no cost: confidence 1, unit inverse-variance weight) is cost 0 with
    the inverse-variance weight off."""
    d = [g.astype(np.float32) for g in (depths if depths is not None else wl.gt_depth)]
    n = [g.astype(np.float32) for g in wl.gt_normal]
    if costs is None:
        costs = [np.zeros(g.shape, np.float32) for g in d]
        kw.setdefault("inverse_variance", 0)
    p = fusion.default_score_fusion(**kw)
    return oracle.fuse_scored(fc, d, n, costs, list(wl.images), range(len(d)), p, threads)


def _ref_error(wl, cl):
    """Relative depth error of each point in its reference view (view and pixel from the point key)."""
    keys = cl.keys.astype(np.int64)
    err = np.empty(len(cl))
    for i in range(len(cl)):
        v, row, col = int(keys[i] >> 32), int((keys[i] >> 16) & 0xFFFF), int(keys[i] & 0xFFFF)
        z = (wl.cams[v].r @ cl.positions[i].astype(np.float64) + wl.cams[v].t)[2]
        err[i] = abs(z - wl.gt_depth[v][row, col]) / wl.gt_depth[v][row, col]
    return err


def test_fuses_true_maps_accurately(scene):
    wl, fc = scene
    cl = _run(wl, fc)
    assert len(cl) > 0.1 * sum(g.size for g in wl.gt_depth)
    assert (cl.vis_counts >= 2).all()  # default tau 2 needs the reference and at least one agreeing view
    keys = cl.keys.astype(np.int64)
    assert (np.diff(keys) > 0).all()  # (view, pixel) order; image ids here are the view indices
    err = _ref_error(wl, cl)
    assert np.median(err) < 0.002 and np.quantile(err, 0.99) < 0.01


def test_mark_used_reduces_duplicates(scene):
    wl, fc = scene
    assert len(_run(wl, fc)) < len(_run(wl, fc, mark_used=0))


def test_point_count_monotone_in_tau(scene):
    wl, fc = scene
    counts = [len(_run(wl, fc, tau=t)) for t in (0.5, 1.5, 2.5, 3.5, 4.5, 5.5, 6.5, 8.5)]
    assert all(b <= a for a, b in zip(counts, counts[1:]))
    assert counts[-1] < counts[0]


def test_free_space_violations_are_rejected(scene):
    """A block of one view pulled toward its camera (depth × 0.6) survives at tau 0.5 without the penalty and is
    rejected with it (λ = 1): the other views see the true surface behind those points."""
    wl, fc = scene
    depth = [g.astype(np.float32).copy() for g in wl.gt_depth]
    depth[4][40:80, 60:100] *= np.float32(0.6)
    floating = lambda cl: int((_ref_error(wl, cl) > 0.2).sum())
    no_pen = _run(wl, fc, depth, tau=0.5, **{"lambda_": 0.0})
    pen = _run(wl, fc, depth, tau=0.5)
    assert floating(no_pen) > 500
    assert floating(pen) == 0


def _noisy(wl):
    rng = np.random.default_rng(11)
    return [(g * (1.0 + rng.uniform(-0.002, 0.002, g.shape))).astype(np.float32) for g in wl.gt_depth]


def test_deterministic_across_threads(scene):
    wl, fc = scene
    depth = _noisy(wl)
    a = _run(wl, fc, depth, threads=1, tau=1.5)
    for t in (2, 4, None):
        b = _run(wl, fc, depth, threads=t, tau=1.5)
        np.testing.assert_array_equal(a.keys, b.keys)
        np.testing.assert_array_equal(a.positions, b.positions)
        np.testing.assert_array_equal(a.normals, b.normals)
        np.testing.assert_array_equal(a.colors, b.colors)
        np.testing.assert_array_equal(a.vis, b.vis)


def _gray(img, x, y):
    h, w = img.shape
    v = np.float32(img[min(y, h - 1), min(x, w - 1)]) * np.float32(255.0)
    return float(min(max(float(np.rint(v)), 0.0), 255.0))


def _python_candidate(fc, depth, normal, cost, imgs, used, p, v, row, col):
    """view_candidates (fusion_score.rs:214-300) for one pixel in Python floats (math.exp / math.acos): None or
    (score, position, normal, colour, sorted views)."""
    T = fc.table
    K = lambda c: list(T[c].k)
    R = lambda c: [list(T[c].r[3 * i:3 * i + 3]) for i in range(3)]
    t_ = lambda c: list(T[c].t)

    def centre(c):
        r, t = R(c), t_(c)
        return [-(r[0][j] * t[0] + r[1][j] * t[1] + r[2][j] * t[2]) for j in range(3)]

    def project(c, x):
        r, t, k = R(c), t_(c), K(c)
        cz = r[2][0] * x[0] + r[2][1] * x[1] + r[2][2] * x[2] + t[2]
        if cz <= 0.0:
            return None
        cx = r[0][0] * x[0] + r[0][1] * x[1] + r[0][2] * x[2] + t[0]
        cy = r[1][0] * x[0] + r[1][1] * x[1] + r[1][2] * x[2] + t[1]
        return k[0] * cx / cz + k[2], k[1] * cy / cz + k[3], cz

    def dir_world(c, q):
        r = R(c)
        return [r[0][i] * q[0] + r[1][i] * q[1] + r[2][i] * q[2] for i in range(3)]

    def backproject(c, cl, rw, d):
        k, t = K(c), t_(c)
        cc = [(cl - k[2]) / k[0] * d, (rw - k[3]) / k[1] * d, d]
        return dir_world(c, [cc[0] - t[0], cc[1] - t[1], cc[2] - t[2]])

    def conf(c, y, x):
        return min(max(1.0 - float(cost[c][y, x]), 0.0), 1.0)

    def inv_var(c, y, x, d):
        if not p.inverse_variance or not T[c].baseline > 0.0:
            return 1.0
        spx = p.sigma_px0 + p.sigma_px_slope * float(min(max(cost[c][y, x], np.float32(0)), np.float32(2)))
        sd = d * d * spx / (K(c)[0] * T[c].baseline)
        return 1.0 / max(sd * sd, 1e-300)

    d = float(depth[v][row, col])
    if not d > 0.0:
        return None
    dot = lambda a, b: a[0] * b[0] + a[1] * b[1] + a[2] * b[2]
    x = backproject(v, float(col), float(row), d)
    nw = dir_world(v, [float(q) for q in normal[v][row, col]])
    cv = centre(v)
    rr = [x[i] - cv[i] for i in range(3)]
    l_ref = math.sqrt(dot(rr, rr))
    s_ref = conf(v, row, col)
    w0 = s_ref * inv_var(v, row, col, d)
    sum_s, sum_p, sw = s_ref, 0.0, w0
    sx = [a * w0 for a in x]
    sn = [a * w0 for a in nw]
    sc = [_gray(imgs[v], col, row) * w0] * 3
    views = {v}
    ov = [o for o in fc.overlap[v] if o != v and used[o]][:p.num_neighbors]
    cos_n = math.cos(math.radians(p.normal_error_deg))
    k_e = 1.0 / (2.0 * p.sigma_e_px * p.sigma_e_px)
    st = math.radians(p.sigma_theta_deg)
    k_t = 1.0 / (2.0 * st * st)
    for j in ov:
        pr = project(j, x)
        if pr is None:
            continue
        u, vv, z = pr
        cu, rv = math.floor(u + 0.5), math.floor(vv + 0.5)
        h, w = depth[j].shape
        if cu < 0 or rv < 0 or cu >= w or rv >= h:
            continue
        od = float(depth[j][rv, cu])
        if od <= 0.0:
            continue
        cj = conf(j, rv, cu)
        if abs(z - od) / od > p.depth_error:
            if z < od * (1.0 - p.depth_error):
                sum_p += cj
            continue
        no = dir_world(j, [float(q) for q in normal[j][rv, cu]])
        if dot(no, nw) < cos_n:
            continue
        xo = backproject(j, float(cu), float(rv), od)
        bp = project(v, xo)
        if bp is None:
            continue
        e2 = (bp[0] - col) ** 2 + (bp[1] - row) ** 2
        cj3 = centre(j)
        rj = [x[i] - cj3[i] for i in range(3)]
        th = math.acos(min(max(dot(rr, rj) / (l_ref * math.sqrt(dot(rj, rj))), -1.0), 1.0))
        s = cj * math.exp(-e2 * k_e) * (1.0 - math.exp(-th * th * k_t))
        sum_s += s
        if s <= 0.0:
            continue
        wo = s * inv_var(j, rv, cu, od)
        co = _gray(imgs[j], cu, rv)
        sw += wo
        for k in range(3):
            sx[k] += wo * xo[k]
            sn[k] += wo * no[k]
            sc[k] += wo * co
        views.add(j)
    score = sum_s - getattr(p, "lambda") * sum_p
    if score < p.tau or not (sw > 0.0 and math.isfinite(sw)):
        return None
    ln = math.sqrt(dot(sn, sn))
    if ln < 1.1920928955078125e-07:
        return None
    colour = [min(max(math.floor(a / sw + 0.5), 0.0), 255.0) for a in sc]  # sums >= 0: half away from zero
    return (score, [a / sw for a in sx], [a / ln for a in sn], colour, sorted(views))


def test_candidates_equal_independent_restatement(scene):
    """Without mark_used the output is every candidate: a sample of pixels of every view, restated in Python with the
    platform's exp / acos, with costs that vary (confidence and the inverse-variance weight both matter)."""
    wl, fc = scene
    rng = np.random.default_rng(4)
    depth = _noisy(wl)
    normal = [g.astype(np.float32) for g in wl.gt_normal]
    cost = [rng.uniform(-0.2, 0.9, g.shape).astype(np.float32) for g in depth]
    imgs = list(wl.images)
    p = fusion.default_score_fusion(mark_used=0, tau=1.2, num_neighbors=4)
    cl = oracle.fuse_scored(fc, depth, normal, cost, imgs, range(len(depth)), p)
    by_key = {int(k): i for i, k in enumerate(cl.keys)}
    used = [True] * len(depth)
    checked = found = 0
    for v in range(len(depth)):
        h, w = depth[v].shape
        for pix in range(v, h * w, 53):
            row, col = divmod(pix, w)
            want = _python_candidate(fc, depth, normal, cost, imgs, used, p, v, row, col)
            if want is not None and abs(want[0] - p.tau) < 1e-9:
                continue  # a score on the threshold itself may fall either way under a 1-ulp exp
            key = (v << 32) | (row << 16) | col
            got = by_key.get(key)
            assert (got is None) == (want is None), (v, row, col)
            checked += 1
            if want is None:
                continue
            found += 1
            np.testing.assert_allclose(cl.positions[got], want[1], rtol=1e-6, atol=1e-6)
            np.testing.assert_allclose(cl.normals[got], want[2], rtol=1e-5, atol=1e-6)
            assert np.all(np.abs(cl.colors[got].astype(int) - np.array(want[3], int)) <= 1)
            assert cl.visibility(got) == want[4]
    assert checked > 2000 and found > 300


def _rounds(pixsets, ranks):
    """The reference's claim rounds (fusion_score.rs:352-414), sequentially: reset, reject-or-claim by minimum rank,
    adopt the candidates holding all their pixels, lock their pixels."""
    FREE, LOCKED = None, 0
    claim = {}
    state = [0] * len(pixsets)
    active = list(range(len(pixsets)))
    while active:
        for g in active:
            for q in pixsets[g]:
                if claim.get(q) != LOCKED:
                    claim[q] = FREE
        for g in active:
            if any(claim.get(q) == LOCKED for q in pixsets[g]):
                state[g] = 2
                continue
            for q in pixsets[g]:
                claim[q] = ranks[g] if claim[q] is FREE else min(claim[q], ranks[g])
        for g in active:
            if state[g] == 0 and all(claim[q] == ranks[g] for q in pixsets[g]):
                state[g] = 1
        for g in active:
            if state[g] == 1:
                for q in pixsets[g]:
                    claim[q] = LOCKED
        active = [g for g in active if state[g] == 0]
    return [s == 1 for s in state]


def _greedy(pixsets, ranks):
    taken, out = set(), [False] * len(pixsets)
    for g in sorted(range(len(pixsets)), key=lambda g: ranks[g]):
        if not any(q in taken for q in pixsets[g]):
            out[g] = True
            taken.update(pixsets[g])
    return out


def _device_rounds(pixsets, ranks, rng):
    """The engine's form of the rounds (k_score_reset / k_score_claim / k_score_adopt): rejection in the reset phase,
    adoption and locking in one phase, the undecided ones compacted into the next round's list in completion order.
    Threads of a phase run one at a time in a random order, each thread's steps interleaved with nothing: every
    pixel's final claim is the same for any order, and the adopt phase's outcome must not depend on it."""
    FREE, LOCKED = 1 << 64, 0
    claim = {}
    state = [2] * len(pixsets)  # 2 undecided, 1 adopted, 0 rejected
    active = list(range(len(pixsets)))
    while active:
        for g in rng.permutation(active).tolist():  # reset: free unlocked pixels, reject on a locked one
            locked = False
            for q in pixsets[g]:
                if claim.get(q, FREE) == LOCKED:
                    locked = True
                else:
                    claim[q] = FREE
            if locked:
                state[g] = 0
        for g in rng.permutation(active).tolist():  # claim: atomic minimum
            if state[g] == 2:
                for q in pixsets[g]:
                    claim[q] = min(claim.get(q, FREE), ranks[g])
        nxt = []
        for g in rng.permutation(active).tolist():  # adopt and lock
            if state[g] != 2:
                continue
            if all(claim[q] == ranks[g] for q in pixsets[g]):
                state[g] = 1
                for q in pixsets[g]:
                    claim[q] = LOCKED
            else:
                nxt.append(g)
        active = nxt
    return [x == 1 for x in state]


@pytest.mark.parametrize("seed", range(8))
def test_claim_rounds_equal_greedy_selection(seed):
    """The reference's rounds and the engine's form of them both choose what greedy selection in priority order
    chooses, on random pixel sets with many overlaps, for several thread orders."""
    rng = np.random.default_rng(seed)
    n, universe = 400, 300 + 100 * seed
    pixsets = [sorted(set(rng.integers(0, universe, size=int(rng.integers(1, 6))).tolist())) for _ in range(n)]
    ranks = (rng.permutation(n) + 1).tolist()
    want = _greedy(pixsets, ranks)
    assert _rounds(pixsets, ranks) == want
    for k in range(3):
        assert _device_rounds(pixsets, ranks, np.random.default_rng(100 * seed + k)) == want


def test_acos64_is_faithful():
    """The viewing-ray angle's arc cosine (a fixed binary64 sequence shared by the engine and the restatement) is
    within 1 ulp of the platform's on [-1, 1]."""
    xs = np.concatenate([np.linspace(-1.0, 1.0, 40001), 1.0 - np.logspace(-16, -1, 2001),
                         -1.0 + np.logspace(-16, -1, 2001), np.logspace(-300, -1, 2001)])
    worst = 0
    for x in xs:
        a, b = oracle.lib().oracle_acos64(float(x)), math.acos(float(x))
        worst = max(worst, abs(int(np.float64(a).view(np.int64)) - int(np.float64(b).view(np.int64))))
    assert worst <= 1


def test_visibility_and_smoothing_after_score_fusion(scene):
    """fuse_depth_maps_with (crates/dense/src/densify.rs:535-556) runs the visibility filter and then the smoothing
    on the score-fusion cloud: the restatement's composed run equals the standalone filter and smoother applied to
    the plain score cloud (overlap lists of the fusion, scene GSD of the fused views)."""
    wl, fc = scene
    rng = np.random.default_rng(8)
    depth = [(g * (1.0 + rng.normal(0, 0.003, g.shape))).astype(np.float32) for g in wl.gt_depth]
    for v in (1, 4):
        depth[v] = depth[v] * np.float32(0.96)  # floaters in front of the surface the other views see
    normal = [g.astype(np.float32) for g in wl.gt_normal]
    cost = [np.full(g.shape, 0.2, np.float32) for g in depth]
    imgs = list(wl.images)
    views = range(len(depth))
    sp = fusion.default_score_fusion(tau=0.5, lambda_=0.0)  # no penalty: the floaters stay candidates
    post = fusion.default_fusion()
    post.visibility_check_views, post.visibility_min_violations, post.visibility_tau = 8, 1, 0.01
    post.smooth_iterations, post.smooth_radius_gsd, post.smooth_sigma_range_gsd = 2, 3.0, 0.5
    plain = oracle.fuse_scored(fc, depth, normal, cost, imgs, views, sp)
    both = oracle.fuse_scored(fc, depth, normal, cost, imgs, views, sp, post=post)
    keep = oracle.filter_visibility(fc, depth, views, plain.positions, [plain.visibility(i) for i in range(len(plain))],
                                    8, 1, 0.01)
    assert 0 < both.visibility_removed == int((~keep).sum()) < len(plain)
    np.testing.assert_array_equal(both.keys, plain.keys[keep])
    np.testing.assert_array_equal(both.normals, plain.normals[keep])
    gs = []
    for g, c in zip(depth, wl.cams):
        s = g.ravel()[g.ravel() > 0][::97].astype(np.float64)
        gs.append(fusion.median_interp(s) / c.k[0])
    smoothed, _ = oracle.smooth(plain.positions[keep], plain.normals[keep], fusion.median_interp(gs), 2, 3.0, 0.5,
                                post.smooth_normal_deg)
    np.testing.assert_array_equal(both.positions, smoothed)
    assert not np.array_equal(smoothed, plain.positions[keep])


def test_views_of_different_sizes():
    """Views of two sizes over one terrain (the reference fuses any mix of view sizes): both fusions keep every key
    inside its own view and put the points of true maps on the surface."""
    a = scenes.formation(96, 72, 1, prefix="a")
    b = scenes.formation(128, 96, 1, prefix="b", y0=2.0)
    cams = a + b
    ext = scenes._extent(cams)
    ia, da, na = scenes.render(a, 4, extent=ext)
    ib, db, nb = scenes.render(b, 4, extent=ext)
    imgs, depth, normal = list(ia) + list(ib), list(da) + list(db), list(na) + list(nb)
    fc = fusion.FusionCams(cams, [[j for j in range(len(cams)) if j != i][:3] for i in range(len(cams))])
    cost = [np.zeros(d.shape, np.float32) for d in depth]
    wl = type("W", (), {"cams": cams, "gt_depth": depth})
    for cl in (oracle.fuse(fc, depth, normal, cost, imgs, range(len(cams)), fusion.default_fusion(2)),
               oracle.fuse_scored(fc, depth, normal, cost, imgs, range(len(cams)),
                                  fusion.default_score_fusion(inverse_variance=0))):
        assert len(cl) > 2000
        keys = cl.keys.astype(np.int64)
        v, row, col = keys >> 32, (keys >> 16) & 0xFFFF, keys & 0xFFFF
        assert ((row < np.array([d.shape[0] for d in depth])[v]) & (col < np.array([d.shape[1] for d in depth])[v])).all()
        assert set(v.tolist()) == set(range(len(cams)))
        err = _ref_error(wl, cl)
        assert np.median(err) < 0.002 and np.quantile(err, 0.99) < 0.01
