"""Post-processing and fusion restatements on the CPU, pinned by the reference's own tests: the speckle known answer
of crates/dense/src/postproc.rs (tests::speckle_and_fill), the PLY layout of crates/dense/tests/host_parts.rs
(ply_output_layout), and the fusion properties of host_parts.rs (fused ground-truth maps lie on the surface; the
result is deterministic; a view whose depth is scaled by 2 % stops merging at the 1 % tolerance)."""
import numpy as np
import pytest

from cumulus3d_b200 import fusion, scenes
from oracle import oracle


def _speckle_case():
    w, h = 40, 30
    d = np.full((h, w), 10.0, np.float32)
    n = np.tile(np.float32([0, 0, -1]), (h, w, 1))
    c = np.full((h, w), 0.5, np.float32)
    for (x, y) in [(5, 5), (6, 5), (5, 6), (6, 6)]:
        d[y, x] = 5.0
    d[20:23, 20:23] = 0.0
    p = fusion.default_post()
    p.speckle_min_area_frac = 10.0 / (w * h)
    return d, n, c, p


def test_speckle_known_answer():
    d, n, c, p = _speckle_case()
    assert oracle.remove_speckles(d, n, c, p) == 4
    assert d[5, 5] == 0.0 and (n[5, 5] == 0).all()
    assert d[0, 0] == 10.0


def test_speckle_keeps_low_cost_components_and_defaults():
    d, n, c, p = _speckle_case()
    c[5:7, 5:7] = 0.1  # median cost 0.1 <= keep 0.2: kept
    assert oracle.remove_speckles(d, n, c, p) == 0
    p = fusion.default_post()
    assert (p.remove_speckles, round(p.speckle_rel_depth, 6), p.speckle_min_area_frac,
            round(p.speckle_keep_cost, 6)) == (1, 0.02, 2e-4, 0.2)
    d, n, c, _ = _speckle_case()
    assert oracle.remove_speckles(d, n, c, p) == 0  # ceil(1200·2e-4) = 1: off


def test_fill_holes_known_answer():
    """speckle_and_fill (crates/dense/src/postproc.rs:208-234): after the 2×2 speckle is erased, hole filling at
    flat gray fills its 4 pixels and the 3×3 hole (13 pixels) with the surrounding depth 10."""
    d, n, c, p = _speckle_case()
    p.fill_holes = 1
    p.fill_max_frac = 0.1
    assert oracle.remove_speckles(d, n, c, p) == 4
    assert d[5, 5] == 0.0
    raw = np.full(d.shape, 0.3, np.float32)
    gray = np.full(d.shape, 100, np.uint8)
    assert oracle.fill_holes(d, n, c, raw, gray, (50.0, 50.0, 19.5, 14.5), p) == 13
    assert abs(float(d[21, 21]) - 10.0) < 1e-4
    assert (d > 0).all() and (n[21, 21] == np.float32([0, 0, -1])).all() and c[21, 21] == np.float32(0.5)


def test_fill_holes_defaults_and_gates():
    p = fusion.default_post()
    assert (p.fill_holes, p.fill_max_frac, round(p.fill_edge_step, 6), p.fill_max_cost) == (0, 0.01, 0.06, 1.0)
    d, n, c, p = _speckle_case()
    p.fill_max_frac = 0.1
    gray = np.full(d.shape, 100, np.uint8)
    # a run cost above fill_max_cost keeps a hole pixel empty; a gray edge (jump > 0.06·255) stops the walk
    raw = np.full(d.shape, 0.3, np.float32)
    raw[21, 21] = 1.5
    gray[:, 23:] = 200
    gray[23:, :] = 200
    gray[:20, :] = 200
    gray[:, :20] = 200
    filled = oracle.fill_holes(d, n, c, raw, gray, (50.0, 50.0, 19.5, 14.5), p)
    assert d[21, 21] == 0.0
    assert filled == 0  # every walk from the hole meets the edge before a valid pixel


def test_gray_round_trip_of_unit_planes():
    """The device derives a pixel's 8-bit gray as round(255·v) from the plane value v = correctly rounded u/255."""
    u = np.arange(256, dtype=np.uint8)
    v = scenes.unit_plane(u.reshape(16, 16)).ravel().astype(np.float32)
    assert (np.rint(v * np.float32(255.0)).astype(np.int64) == np.arange(256)).all()


def test_speckle_components_do_not_depend_on_scan_order():
    rng = np.random.default_rng(3)
    d = rng.choice([0.0, 10.0, 10.1, 13.0], size=(48, 64), p=[0.3, 0.3, 0.2, 0.2]).astype(np.float32)
    c = rng.uniform(0, 1, d.shape).astype(np.float32)
    p = fusion.default_post()
    p.speckle_min_area_frac = 0.005
    a, na = d.copy(), np.zeros(d.shape + (3,), np.float32)
    b, nb = d[::-1, ::-1].copy(), np.zeros(d.shape + (3,), np.float32)
    ra = oracle.remove_speckles(a, na, c, p)
    rb = oracle.remove_speckles(b, nb, c[::-1, ::-1].copy(), p)
    assert ra == rb > 0
    np.testing.assert_array_equal(a, b[::-1, ::-1])


def test_ply_layout_matches_reference(tmp_path):
    f = tmp_path / "a.ply"
    pos = np.float32([[1, 2, 3], [4, 5, 6]])
    nrm = np.float32([[0, 0, 1], [0, 0, 1]])
    col = np.uint8([[1, 2, 3], [4, 5, 6]])
    fusion.write_ply(f, pos, nrm, col)
    b = f.read_bytes()
    hdr = ("ply\nformat binary_little_endian 1.0\nelement vertex 2\nproperty float x\nproperty float y\n"
           "property float z\nproperty float nx\nproperty float ny\nproperty float nz\nproperty uchar red\n"
           "property uchar green\nproperty uchar blue\nend_header\n").encode()
    assert b[:len(hdr)] == hdr
    assert len(b) - len(hdr) == 54
    rec = np.frombuffer(b[len(hdr):], dtype=np.dtype([("p", "<f4", 3), ("n", "<f4", 3), ("c", "u1", 3)]))
    np.testing.assert_array_equal(rec["p"], pos)
    np.testing.assert_array_equal(rec["c"], col)


@pytest.fixture(scope="module")
def gt_scene():
    wl = scenes.workload_small(160, 120, views=6, window_radius=3, seed=3, positions=2)
    src = [list(kv.sources) for kv in wl.input.views]
    return wl, fusion.FusionCams(wl.cams, src)


def _fuse_gt(wl, fc, depths=None, threads=None, min_views=3):
    d = [g.astype(np.float32) for g in (depths if depths is not None else wl.gt_depth)]
    n = [g.astype(np.float32) for g in wl.gt_normal]
    c = [np.full(g.shape, 0.3, np.float32) for g in d]
    return oracle.fuse(fc, d, n, c, list(wl.images), range(len(d)), fusion.default_fusion(min_views), threads)


def test_fusion_of_true_maps_lies_on_surfaces(gt_scene):
    wl, fc = gt_scene
    cl = _fuse_gt(wl, fc)
    assert len(cl) > 0.05 * sum(g.size for g in wl.gt_depth)
    assert (cl.vis_counts >= 4).all()  # reference + at least 3 agreeing views
    keys = cl.keys.astype(np.int64)
    assert (np.diff(keys) > 0).all()  # reference order: ascending keys
    err = []
    for i in range(0, len(cl), 37):
        v, row, col = int(keys[i] >> 32), int((keys[i] >> 16) & 0xFFFF), int(keys[i] & 0xFFFF)
        pc = wl.cams[v].r @ cl.positions[i].astype(np.float64) + wl.cams[v].t
        err.append(abs(pc[2] - wl.gt_depth[v][row, col]) / wl.gt_depth[v][row, col])
    assert np.max(err) < 0.01 and np.median(err) < 0.002
    again = _fuse_gt(wl, fc, threads=1)
    np.testing.assert_array_equal(again.keys, cl.keys)
    np.testing.assert_array_equal(again.positions, cl.positions)


def test_fusion_depth_tolerance(gt_scene):
    wl, fc = gt_scene
    base = _fuse_gt(wl, fc)
    scaled = [g.copy() for g in wl.gt_depth]
    scaled[2] = scaled[2] * 1.02
    sc = _fuse_gt(wl, fc, scaled)
    merged = lambda cl: int(sum(1 for i in range(len(cl)) if 2 in cl.visibility(i) and cl.vis_counts[i] > 1))
    assert merged(sc) * 50 < merged(base)


def _rotated_normals(normals, deg):
    """Every normal turned by exactly `deg` (Rodrigues rotation about an axis perpendicular to it)."""
    n = normals.astype(np.float64)
    k = np.cross(n, np.array([1.0, 0.0, 0.0]))
    k /= np.linalg.norm(k, axis=-1, keepdims=True)
    a = np.radians(deg)
    return (n * np.cos(a) + np.cross(k, n) * np.sin(a)).astype(np.float32)


def test_fusion_normal_tolerance_and_marks(gt_scene):
    """fusion_depth_and_normal_tolerances (normal half) and consistency_fusion_of_true_maps (crates/dense/tests/
    host_parts.rs:163-196, :231-250): one view's normals turned by 15° stop merging at the 10° tolerance, by 8° they
    still merge; without marks the same surface is emitted again per view (more points)."""
    wl, fc = gt_scene
    d = [g.astype(np.float32) for g in wl.gt_depth]
    c = [np.full(g.shape, 0.3, np.float32) for g in d]
    prm = fusion.default_fusion(3)

    def run(normals, p=prm):
        return oracle.fuse(fc, d, normals, c, list(wl.images), range(len(d)), p)

    merged = lambda cl: int(sum(1 for i in range(len(cl)) if 2 in cl.visibility(i) and cl.vis_counts[i] > 1))
    n0 = [g.astype(np.float32) for g in wl.gt_normal]
    base = run(n0)
    for deg, far in ((15.0, True), (8.0, False)):
        nr = [g.copy() for g in n0]
        nr[2] = _rotated_normals(nr[2], deg)
        m = merged(run(nr))
        assert (m * 20 < merged(base)) if far else (m * 2 > merged(base)), deg
    nomark = fusion.default_fusion(3)
    nomark.mark_used = 0
    assert len(run(n0, nomark)) > len(base)


def _fuse_gt_noisy(wl, fc, prm, seed=5):
    """Ground-truth maps with multiplicative depth noise, so the first pass leaves pixels for the second."""
    rng = np.random.default_rng(seed)
    d = [(g * (1.0 + rng.normal(0, 0.006, g.shape))).astype(np.float32) for g in wl.gt_depth]
    n = [g.astype(np.float32) for g in wl.gt_normal]
    c = [np.full(g.shape, 0.3, np.float32) for g in d]
    return oracle.fuse(fc, d, n, c, list(wl.images), range(len(d)), prm)


def test_residual_release_equals_none_and_second_pass_appends(gt_scene):
    """FusionResidual (crates/dense/src/fusion.rs:210-218): Release gives the None result; SecondPass keeps the
    first-pass points as they are and appends its own, in ascending key, none of them within min_dist_gsd × GSD of a
    first-pass point, each from a distinct reference pixel."""
    wl, fc = gt_scene
    base = fusion.default_fusion(3)
    none = _fuse_gt_noisy(wl, fc, base)
    rel = fusion.default_fusion(3)
    rel.residual = 1
    release = _fuse_gt_noisy(wl, fc, rel)
    np.testing.assert_array_equal(release.keys, none.keys)
    np.testing.assert_array_equal(release.positions, none.positions)
    sp = fusion.default_fusion(3)
    sp.residual = 2
    two = _fuse_gt_noisy(wl, fc, sp)
    n1 = len(two) - two.residual
    assert n1 == len(none) and two.residual > 0
    np.testing.assert_array_equal(two.keys[:n1], none.keys)
    np.testing.assert_array_equal(two.positions[:n1], none.positions)
    k2 = two.keys[n1:].astype(np.int64)
    assert (np.diff(k2) > 0).all()
    assert not np.isin(two.keys[n1:], none.keys).any()
    assert (two.vis_counts[n1:] >= 3).all()  # reference + residual_min_views (2)
    # the distance rule, with the GSD the restatement uses: the median over views of the median valid depth / fx
    d1 = two.positions[:n1].astype(np.float64)
    d2 = two.positions[n1:].astype(np.float64)
    gsd_lo = 0.5 * min(np.median(g[g > 0]) / c.k[0] for g, c in zip(wl.gt_depth, wl.cams)) * 0.9
    for x in d2[::7]:
        assert np.min(np.sum((d1 - x) ** 2, axis=1)) > gsd_lo ** 2


def test_fusion_keys_unique_reproducible_and_thread_independent(gt_scene):
    """fusion_keys_are_unique_and_reproducible and second_pass_is_deterministic (crates/dense/tests/
    residual_fusion.rs:154-200): consistency fusion, its second pass and score fusion give unique keys whose view
    and pixel exist, the same cloud on 1, 3 and all threads, and the same keys when run again."""
    wl, fc = gt_scene
    rng = np.random.default_rng(5)
    d = [(g * (1.0 + rng.normal(0, 0.006, g.shape))).astype(np.float32) for g in wl.gt_depth]
    n = [g.astype(np.float32) for g in wl.gt_normal]
    c = [np.full(g.shape, 0.3, np.float32) for g in d]
    sp = fusion.default_fusion(3)
    sp.residual = 2
    args = (fc, d, n, c, list(wl.images), range(len(d)))
    runs = {"consistency": lambda t: oracle.fuse(*args, fusion.default_fusion(3), t),
            "second pass": lambda t: oracle.fuse(*args, sp, t),
            "score": lambda t: oracle.fuse_scored(*args, fusion.default_score_fusion(), t)}
    for name, run in runs.items():
        a = run(None)
        assert len(a) > 500, name
        assert len(set(a.keys.tolist())) == len(a), name
        for t in (1, 3):
            b = run(t)
            np.testing.assert_array_equal(a.keys, b.keys, name)
            np.testing.assert_array_equal(a.positions, b.positions, name)
            np.testing.assert_array_equal(a.normals, b.normals, name)
            np.testing.assert_array_equal(a.colors, b.colors, name)
            np.testing.assert_array_equal(a.vis, b.vis, name)
        keys = a.keys.astype(np.int64)
        img, row, col = keys >> 32, (keys >> 16) & 0xFFFF, keys & 0xFFFF
        assert ((img >= 0) & (img < len(d))).all(), name  # image ids here are the view indices
        h = np.array([g.shape[0] for g in d])[img]
        w = np.array([g.shape[1] for g in d])[img]
        assert ((row < h) & (col < w)).all(), name


def test_residual_ply_holds_the_second_pass_points(gt_scene, tmp_path):
    """DenseOutput::write_ply / write_residual_ply (crates/dense/src/densify.rs:143-180): the parent folder is
    created; the residual file holds exactly the second-pass points; without them nothing is written."""
    wl, fc = gt_scene
    sp = fusion.default_fusion(3)
    sp.residual = 2
    cl = _fuse_gt_noisy(wl, fc, sp)
    r = cl.num_residual()
    assert r > 0
    f = tmp_path / "out" / "dense" / "residual.ply"
    assert cl.write_residual_ply(f)
    b = f.read_bytes()
    body = b[b.index(b"end_header\n") + len(b"end_header\n"):]
    rec = np.frombuffer(body, dtype=np.dtype([("p", "<f4", 3), ("n", "<f4", 3), ("c", "u1", 3)]))
    assert len(rec) == r and f"element vertex {r}\n".encode() in b
    np.testing.assert_array_equal(rec["p"], cl.positions[len(cl) - r:])
    np.testing.assert_array_equal(rec["c"], cl.colors[len(cl) - r:])
    cl.write_ply(tmp_path / "x" / "all.ply")
    a = (tmp_path / "x" / "all.ply").read_bytes()
    assert len(a) - (a.index(b"end_header\n") + len(b"end_header\n")) == 27 * len(cl)
    none = _fuse_gt_noisy(wl, fc, fusion.default_fusion(3))
    assert none.num_residual() == 0
    assert not none.write_residual_ply(tmp_path / "none.ply") and not (tmp_path / "none.ply").exists()


def _visibility_keep_py(cloud, depths, fc_views, used, limit, tau, min_viol):
    """filter_visibility (crates/dense/src/visibility.rs:106-151) restated in Python: the keep flag of every point."""
    keep = []
    for i in range(len(cloud)):
        x = cloud.positions[i].astype(np.float64)
        cand = []
        full = False
        for v in cloud.visibility(i):
            if full:
                break
            for o in fc_views[v]["overlap"]:
                if len(cand) >= limit:
                    full = True
                    break
                if o not in cand:
                    cand.append(o)
        viol = sup = 0
        for v in cand:
            if not used[v]:
                continue
            c = fc_views[v]
            pc = c["r"] @ x + c["t"]
            if pc[2] <= 0:
                continue
            col = np.round(c["k"][0] * pc[0] / pc[2] + c["k"][2])
            row = np.round(c["k"][1] * pc[1] / pc[2] + c["k"][3])
            h, w = depths[v].shape
            if col < 0 or row < 0 or col >= w or row >= h:
                continue
            dv = float(depths[v][int(row), int(col)])
            if dv <= 0:
                continue
            if pc[2] < dv * (1 - tau):
                viol += 1
            elif abs(pc[2] - dv) <= tau * dv:
                sup += 1
        keep.append(not (viol >= min_viol and viol > sup))
    return np.array(keep, bool)


def test_visibility_filter_matches_independent_restatement(gt_scene):
    """Four of six views see 5 % too far: points fused from the other two violate free space in those four."""
    wl, fc = gt_scene
    d = [g.astype(np.float32) for g in wl.gt_depth]
    for v in (2, 3, 4, 5):
        d[v] = d[v] * np.float32(1.05)
    n = [g.astype(np.float32) for g in wl.gt_normal]
    c = [np.full(g.shape, 0.3, np.float32) for g in d]
    prm = fusion.default_fusion(1)
    base = oracle.fuse(fc, d, n, c, list(wl.images), range(len(d)), prm)
    prm.visibility_check_views, prm.visibility_min_violations, prm.visibility_tau = 8, 2, 0.01
    filt = oracle.fuse(fc, d, n, c, list(wl.images), range(len(d)), prm)
    views = []
    for v, cam in enumerate(wl.cams):
        views.append({"k": cam.k, "r": cam.r, "t": cam.t, "overlap": [int(o) for o in fc.overlap[v]]})
    keep = _visibility_keep_py(base, d, views, [True] * len(d), 8, 0.01, 2)
    assert filt.visibility_removed == int((~keep).sum()) > 0
    np.testing.assert_array_equal(filt.keys, base.keys[keep])
    np.testing.assert_array_equal(filt.positions, base.positions[keep])


def test_exp64_is_faithful():
    """The smoothing weights' exponential (a fixed binary64 sequence shared by the engine and the restatement) is
    within 1 ulp of the platform's over the arguments the weights take and beyond."""
    import math
    xs = np.concatenate([np.linspace(-745.0, 0.0, 20001), -np.logspace(-12, 2, 4001), np.linspace(0.0, 700.0, 2001)])
    worst = 0
    for x in xs:
        a, b = oracle.lib().oracle_exp64(float(x)), math.exp(float(x))
        if b == 0.0 or not math.isfinite(b):
            continue
        worst = max(worst, abs(int(np.float64(a).view(np.int64)) - int(np.float64(b).view(np.int64))))
    assert worst <= 1


def test_smoothing_moves_points_along_normals_toward_the_surface(gt_scene):
    """smooth_along_normals (crates/dense/src/smooth.rs:143-220): keys and normals stay, every point moves along its
    own normal only, and noisy depths end up closer to the true surface."""
    wl, fc = gt_scene
    rng = np.random.default_rng(9)
    d = [(g * (1.0 + rng.normal(0, 0.002, g.shape))).astype(np.float32) for g in wl.gt_depth]
    n = [g.astype(np.float32) for g in wl.gt_normal]
    c = [np.full(g.shape, 0.3, np.float32) for g in d]
    prm = fusion.default_fusion(2)
    prm.max_depth_error = 0.02
    base = oracle.fuse(fc, d, n, c, list(wl.images), range(len(d)), prm)
    prm.smooth_iterations, prm.smooth_radius_gsd = 2, 3.0
    sm = oracle.fuse(fc, d, n, c, list(wl.images), range(len(d)), prm)
    np.testing.assert_array_equal(sm.keys, base.keys)
    np.testing.assert_array_equal(sm.normals, base.normals)
    mv = sm.positions.astype(np.float64) - base.positions.astype(np.float64)
    nn = base.normals.astype(np.float64)
    nn /= np.linalg.norm(nn, axis=1, keepdims=True)
    tang = mv - (mv * nn).sum(1, keepdims=True) * nn
    assert np.abs(tang).max() < 1e-4 and np.abs(mv).max() > 0

    def err(cloud):
        e = []
        keys = cloud.keys.astype(np.int64)
        for i in range(0, len(cloud), 11):
            v, row, col = int(keys[i] >> 32), int((keys[i] >> 16) & 0xFFFF), int(keys[i] & 0xFFFF)
            pc = wl.cams[v].r @ cloud.positions[i].astype(np.float64) + wl.cams[v].t
            e.append(abs(pc[2] - wl.gt_depth[v][row, col]))
        return float(np.median(e))

    assert err(sm) < 0.8 * err(base)


def _mix64(z):
    """mix64 (crates/dense/src/math.rs:40-47): the splitmix64 finalizer."""
    m = (1 << 64) - 1
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def _noisy_plane(n, noise):
    """noisy_plane of crates/dense/src/smooth.rs:231-245: points uniform on [0, 4]² with z uniform in ±noise, normals
    +z, from the reference's mix64 sequence."""
    s = 0x12345678
    vals = np.empty(3 * n)
    for i in range(3 * n):
        s = _mix64((s + 0x9E3779B97F4A7C15) & ((1 << 64) - 1))
        vals[i] = (s >> 11) / float(1 << 53)
    v = vals.reshape(n, 3)
    pos = np.stack([v[:, 0] * 4.0, v[:, 1] * 4.0, (v[:, 2] - 0.5) * 2.0 * noise], 1).astype(np.float32)
    return pos, np.tile(np.float32([0, 0, 1]), (n, 1))


def test_smoothing_thins_a_noisy_plane_without_moving_tangentially():
    """thins_a_noisy_plane_without_moving_tangentially (crates/dense/src/smooth.rs:252-263)."""
    pos, nrm = _noisy_plane(20000, 0.01)
    out, disp = oracle.smooth(pos, nrm, 0.05, 1, 4.0, 1.0, 30.0)
    rms = lambda p: float(np.sqrt(np.mean(p[:, 2].astype(np.float64) ** 2)))
    assert disp > 0.0
    assert rms(out) < 0.5 * rms(pos)
    np.testing.assert_array_equal(out[:, :2], pos[:, :2])


def test_smoothing_keeps_a_step_and_respects_normals():
    """keeps_a_step_and_respects_normals (crates/dense/src/smooth.rs:265-284): two sheets 0.5 apart stay apart under
    the range term; smoothing off leaves a cloud untouched."""
    lower, nrm = _noisy_plane(10000, 0.0)
    upper = lower.copy()
    upper[:, 2] = 0.5
    out, _ = oracle.smooth(np.concatenate([lower, upper]), np.concatenate([nrm, nrm]), 0.05, 2, 12.0, 0.5, 30.0)
    assert (np.abs(out[:10000, 2]) < 1e-4).all()
    assert (np.abs(out[10000:, 2] - 0.5) < 1e-4).all()
    c, cn = _noisy_plane(100, 0.01)
    same, d = oracle.smooth(c, cn, 0.05, 0, 1.0, 0.25, 30.0)  # SmoothParams::default(): 0 iterations
    assert d == 0.0
    np.testing.assert_array_equal(same, c)


def _floater_cloud(wl):
    """setup() of crates/dense/src/visibility.rs:170-189 on this package's scene: five pixels near the middle of view
    0 lifted at their true depth and at 80 % of it (the reference's half depth leaves this scene's narrower frames),
    each point seen by view 0 only; every other view overlaps."""
    cam = wl.cams[0]
    h, w = wl.gt_depth[0].shape
    pix = [(w // 2 + dx, h // 2 + dy) for dx, dy in ((-20, -10), (0, 0), (20, 10), (-10, 15), (10, -15))]
    pts = []
    for frac in (1.0, 0.8):
        for col, row in pix:
            d = float(wl.gt_depth[0][row, col])
            c = np.array([(col - cam.k[2]) / cam.k[0] * d * frac, (row - cam.k[3]) / cam.k[1] * d * frac, d * frac])
            pts.append(cam.r.T @ (c - cam.t))
    n = len(wl.cams)
    overlap = [[o for o in range(n) if o != v] for v in range(n)]
    return np.array(pts, np.float32), [[0]] * len(pts), overlap


def test_visibility_removes_floaters_and_keeps_surface(gt_scene):
    """removes_floaters_and_keeps_plane and default_params_leave_cloud_unchanged (crates/dense/src/visibility.rs:196-
    220): with 8 views, 2 violations and 1 % the five floaters go and the five surface points stay; the default
    parameters (check_views 0) keep everything."""
    wl, _ = gt_scene
    pts, vis, overlap = _floater_cloud(wl)
    fc = fusion.FusionCams(wl.cams, [list(kv.sources) for kv in wl.input.views], overlap=overlap)
    depth = [g.astype(np.float32) for g in wl.gt_depth]
    keep = oracle.filter_visibility(fc, depth, range(len(depth)), pts, vis, 8, 2, 0.01)
    assert keep.tolist() == [True] * 5 + [False] * 5
    p = fusion.default_fusion()
    keep = oracle.filter_visibility(fc, depth, range(len(depth)), pts, vis, p.visibility_check_views,
                                    p.visibility_min_violations, p.visibility_tau)
    assert keep.all()


def test_fuse_depth_maps_with_dispatch():
    """fusion.fuse_depth_maps_with picks the fusion as the reference's does (score options present: score fusion with
    the fusion parameters' visibility and smoothing after it; otherwise consistency fusion)."""
    calls = []

    class Session:
        def fuse_resident(self, level, views, cams, p):
            calls.append(("consistency", level, list(views), p.min_consistent_views))

        def fuse_scored_resident(self, level, views, cams, s, post=None):
            calls.append(("score", level, list(views), s.tau, post.smooth_iterations))

        def fused_points(self):
            return "cloud"

    prm = fusion.default_fusion(4)
    prm.smooth_iterations = 2
    assert fusion.fuse_depth_maps_with(Session(), 1, [0, 2], None, prm) == "cloud"
    assert fusion.fuse_depth_maps_with(Session(), 0, [1], None, prm, fusion.default_score_fusion(tau=3.0)) == "cloud"
    assert calls == [("consistency", 1, [0, 2], 4), ("score", 0, [1], 3.0, 2)]


def test_smoothing_equals_direct_restatement():
    """smooth_along_normals (crates/dense/src/smooth.rs:143-220) restated directly in Python (all pairs within the
    radius, the platform's exp) on a small curved, noisy cloud with tilted normals: the restatement's positions agree
    to float32 rounding."""
    rng = np.random.default_rng(12)
    n = 600
    xy = rng.uniform(0, 2, (n, 2))
    z = 0.1 * np.sin(2 * xy[:, 0]) + rng.normal(0, 0.01, n)
    pos = np.column_stack([xy, z]).astype(np.float32)
    nrm = np.column_stack([-0.2 * np.cos(2 * xy[:, 0]), np.zeros(n), np.ones(n)]) + rng.normal(0, 0.05, (n, 3))
    nrm[::50] = 0.0  # normals of length 0 stay put
    nrm = nrm.astype(np.float32)
    gsd, it, rad, srg, deg = 0.02, 2, 6.0, 1.0, 30.0
    got, _ = oracle.smooth(pos, nrm, gsd, it, rad, srg, deg)
    r = rad * gsd
    r2, inv_2ss, inv_2sr = r * r, 1.0 / (2.0 * (0.5 * r) ** 2), 1.0 / (2.0 * (srg * gsd) ** 2)
    cos_n = np.cos(np.radians(deg))
    nn = nrm.astype(np.float64)
    ln = np.linalg.norm(nn, axis=1, keepdims=True)
    nn = np.where(ln > 1e-12, nn / np.where(ln > 0, ln, 1), 0.0)
    cur = pos.copy()
    for _ in range(it):
        p64 = cur.astype(np.float64)
        nxt = np.empty_like(cur)
        for i in range(n):
            ni = nn[i]
            t = 0.0
            if ni.any():
                dv = p64 - p64[i]
                d2 = (dv ** 2).sum(1)
                ok = (d2 <= r2) & (np.arange(n) != i) & (nn @ ni >= cos_n)
                dn = dv[ok] @ ni
                w = np.exp(-d2[ok] * inv_2ss - dn * dn * inv_2sr)
                t = float((w * dn).sum() / (1.0 + w.sum()))
            nxt[i] = (p64[i] + t * ni).astype(np.float32)
        cur = nxt
    np.testing.assert_allclose(got, cur, rtol=0, atol=2e-6)
    assert np.abs(got - pos).max() > 1e-3  # it moved
    np.testing.assert_array_equal(got[::50], pos[::50])


def _consistency_point_py(fc, depth, normal, cost, imgs, p, v, row, col):
    """ConsCtx::evaluate (crates/dense/src/fusion.rs:390-459) for one pixel in Python floats: None or (position,
    normal, colour, sorted views), under FusionParams p (the first consistency_num_images used partners)."""
    import math
    T = fc.table
    R = lambda c: [list(T[c].r[3 * i:3 * i + 3]) for i in range(3)]

    def project(c, x):
        r, t, k = R(c), list(T[c].t), list(T[c].k)
        cz = r[2][0] * x[0] + r[2][1] * x[1] + r[2][2] * x[2] + t[2]
        if cz <= 0.0:
            return None
        cx = r[0][0] * x[0] + r[0][1] * x[1] + r[0][2] * x[2] + t[0]
        cy = r[1][0] * x[0] + r[1][1] * x[1] + r[1][2] * x[2] + t[1]
        return k[0] * cx / cz + k[2], k[1] * cy / cz + k[3], cz

    def world(c, q):
        r = R(c)
        return [r[0][i] * q[0] + r[1][i] * q[1] + r[2][i] * q[2] for i in range(3)]

    def backproject(c, cl, rw, d):
        k, t = list(T[c].k), list(T[c].t)
        cc = [(cl - k[2]) / k[0] * d, (rw - k[3]) / k[1] * d, d]
        return world(c, [cc[0] - t[0], cc[1] - t[1], cc[2] - t[2]])

    def inv_var(c, y, x, d):
        if not p.inverse_variance or not T[c].baseline > 0.0:
            return 1.0
        spx = p.sigma_px0 + p.sigma_px_slope * float(min(max(cost[c][y, x], np.float32(0)), np.float32(2)))
        sd = d * d * spx / (T[c].k[0] * T[c].baseline)
        return 1.0 / max(sd * sd, 1e-300)

    def gray(c, x, y):
        return float(np.rint(np.float32(imgs[c][y, x]) * np.float32(255.0)))

    d = float(depth[v][row, col])
    x = backproject(v, float(col), float(row), d)
    nw = world(v, [float(q) for q in normal[v][row, col]])
    w0 = inv_var(v, row, col, d)
    sw, sx, sn, sc = w0, [a * w0 for a in x], [a * w0 for a in nw], [gray(v, col, row) * w0] * 3
    views = {v}
    hits = 0
    cos_n = math.cos(math.radians(p.max_normal_error_deg))
    for o in [o for o in fc.overlap[v] if o != v][:p.consistency_num_images]:
        pr = project(o, x)
        if pr is None:
            continue
        cu, rv = math.floor(pr[0] + 0.5), math.floor(pr[1] + 0.5)
        h, w = depth[o].shape
        if cu < 0 or rv < 0 or cu >= w or rv >= h:
            continue
        od = float(depth[o][rv, cu])
        if od <= 0.0 or abs(pr[2] - od) / od > p.max_depth_error:
            continue
        xo = backproject(o, float(cu), float(rv), od)
        bp = project(v, xo)
        if bp is None or (bp[0] - col) ** 2 + (bp[1] - row) ** 2 > p.max_reproj_error ** 2:
            continue
        no = world(o, [float(q) for q in normal[o][rv, cu]])
        if no[0] * nw[0] + no[1] * nw[1] + no[2] * nw[2] < cos_n:
            continue
        wo = inv_var(o, rv, cu, od)
        co = gray(o, cu, rv)
        sw += wo
        for k in range(3):
            sx[k] += wo * xo[k]
            sn[k] += wo * no[k]
            sc[k] += wo * co
        views.add(o)
        hits += 1
    ln = math.sqrt(sn[0] ** 2 + sn[1] ** 2 + sn[2] ** 2)
    if hits < p.min_consistent_views or ln < 1.1920928955078125e-07:
        return None
    return [a / sw for a in sx], [a / ln for a in sn], [math.floor(a / sw + 0.5) for a in sc], sorted(views)


def test_consistency_points_equal_independent_restatement(gt_scene):
    """Without marks every pixel is fused on its own: a sample of pixels of every view restated in Python, with
    noisy depths, varying costs (inverse-variance weights) and the default tolerances."""
    wl, fc = gt_scene
    rng = np.random.default_rng(21)
    depth = [(g * (1.0 + rng.normal(0, 0.003, g.shape))).astype(np.float32) for g in wl.gt_depth]
    normal = [g.astype(np.float32) for g in wl.gt_normal]
    cost = [rng.uniform(0.0, 1.2, g.shape).astype(np.float32) for g in depth]
    imgs = list(wl.images)
    p = fusion.default_fusion(2)
    p.mark_used = 0
    cl = oracle.fuse(fc, depth, normal, cost, imgs, range(len(depth)), p)
    by_key = {int(k): i for i, k in enumerate(cl.keys)}
    checked = found = 0
    for v in range(len(depth)):
        h, w = depth[v].shape
        for pix in range(v, h * w, 41):
            row, col = divmod(pix, w)
            if not depth[v][row, col] > 0:
                continue
            want = _consistency_point_py(fc, depth, normal, cost, imgs, p, v, row, col)
            got = by_key.get((v << 32) | (row << 16) | col)
            assert (got is None) == (want is None), (v, row, col)
            checked += 1
            if want is None:
                continue
            found += 1
            np.testing.assert_allclose(cl.positions[got], want[0], rtol=1e-6, atol=1e-6)
            np.testing.assert_allclose(cl.normals[got], want[1], rtol=1e-5, atol=1e-6)
            assert np.all(np.abs(cl.colors[got].astype(int) - np.array(want[2], int)) <= 1)
            assert cl.visibility(got) == want[3]
    assert checked > 2000 and found > 500
