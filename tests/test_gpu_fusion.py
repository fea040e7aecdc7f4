"""Speckle removal and consistency fusion on the GPU against the CPU oracle, bit for bit (zero tolerance: integer
labels and comparisons, and FP64 fusion arithmetic in the same operation order on both sides)."""
import numpy as np
import pytest

from cumulus3d_b200 import fusion, scenes
from cumulus3d_b200.patchstereo import PatchMatchBackend
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pipeline():
    """A short full schedule on 6 views (2 formation stations), read out on the device."""
    wl = scenes.workload_small(160, 120, views=6, window_radius=3, seed=21, iters=2, sources=4, positions=2)
    views = list(range(len(wl.cams)))
    be = PatchMatchBackend(0, math="parity")
    s = be.begin(wl.input)
    s.schedule_resident(views, 2, 1, 1, graph=False)
    s.synchronize()
    yield wl, views, s
    s.close()
    be.close()


def _speckles_ref(states, post):
    out, removed = [], 0
    for st in states:
        d = st.depth.copy()
        n = st.normal.copy()
        removed += oracle.remove_speckles(d, n, st.cost, post)
        out.append((d, n))
    return out, removed


@pytest.mark.parametrize("frac", [2e-4, 0.01])
def test_speckles_bitwise_vs_oracle(pipeline, frac):
    wl, views, s = pipeline
    before = s.readout_resident(views)
    post = fusion.default_post()
    post.speckle_min_area_frac = frac
    want, n_ref = _speckles_ref(before, post)
    n = s.postprocess_resident(0, views, post)
    got = s.readout_download(0, views)
    assert n == n_ref
    if frac == 0.01:
        assert n > 0  # the case removes something
    for g, (d, nn) in zip(got, want):
        np.testing.assert_array_equal(g.depth, d)
        np.testing.assert_array_equal(g.normal, nn)


def test_fusion_bitwise_vs_oracle(pipeline):
    wl, views, s = pipeline
    s.readout_resident(views, download=False)
    s.postprocess_resident(0, views)
    states = s.readout_download(0, views)
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    prm = fusion.default_fusion(3)
    n = s.fuse_resident(0, views, fc, prm)
    got = s.fused_points()
    want = oracle.fuse(fc, [st.depth for st in states], [st.normal for st in states], [st.cost for st in states],
                       [scenes.unit_plane(kv.levels[0].pixels) for kv in wl.input.views], views, prm)
    assert n == len(want) > 0
    np.testing.assert_array_equal(got.keys, want.keys)
    np.testing.assert_array_equal(got.positions, want.positions)
    np.testing.assert_array_equal(got.normals, want.normals)
    np.testing.assert_array_equal(got.colors, want.colors)
    np.testing.assert_array_equal(got.vis_counts, want.vis_counts)
    for i in range(len(want)):
        assert got.visibility(i) == want.visibility(i)
    # the subset without view 0 (view 0's pixels neither references nor partners)
    n2 = s.fuse_resident(0, views[1:], fc, prm)
    want2 = oracle.fuse(fc, [st.depth for st in states], [st.normal for st in states], [st.cost for st in states],
                        [scenes.unit_plane(kv.levels[0].pixels) for kv in wl.input.views], views[1:], prm)
    assert n2 == len(want2)
    np.testing.assert_array_equal(s.fused_points().keys, want2.keys)


def test_second_pass_fusion_bitwise_vs_oracle(pipeline):
    """FusionResidual::SecondPass (crates/dense/src/fusion.rs:540-627) on the device against the restatement: the
    whole cloud (first pass, then the second-pass points) and the residual count equal; Release equals None."""
    wl, views, s = pipeline
    s.readout_resident(views, download=False)
    s.postprocess_resident(0, views)
    states = s.readout_download(0, views)
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    imgs = [scenes.unit_plane(kv.levels[0].pixels) for kv in wl.input.views]
    args = ([st.depth for st in states], [st.normal for st in states], [st.cost for st in states], imgs, views)
    prm = fusion.default_fusion(3)
    prm.residual = 2
    n = s.fuse_resident(0, views, fc, prm)
    got = s.fused_points()
    want = oracle.fuse(fc, *args, prm)
    assert n == len(want) and s.fused_residual == want.residual > 0
    np.testing.assert_array_equal(got.keys, want.keys)
    np.testing.assert_array_equal(got.positions, want.positions)
    np.testing.assert_array_equal(got.normals, want.normals)
    np.testing.assert_array_equal(got.colors, want.colors)
    np.testing.assert_array_equal(got.vis_counts, want.vis_counts)
    for i in range(len(want)):
        assert got.visibility(i) == want.visibility(i)
    # explicit residual tolerances and no distance rule
    prm.residual_depth_error, prm.residual_normal_error_deg, prm.residual_min_dist_gsd = 0.004, 6.0, 0.0
    n2 = s.fuse_resident(0, views, fc, prm)
    want2 = oracle.fuse(fc, *args, prm)
    assert n2 == len(want2) and s.fused_residual == want2.residual
    np.testing.assert_array_equal(s.fused_points().keys, want2.keys)
    rel = fusion.default_fusion(3)
    rel.residual = 1
    n_rel = s.fuse_resident(0, views, fc, rel)
    n_none = s.fuse_resident(0, views, fc, fusion.default_fusion(3))
    assert n_rel == n_none and s.fused_residual == 0


@pytest.mark.parametrize("opts", [{}, {"mark_used": 0}, {"tau": 0.5, "num_neighbors": 3},
                                  {"tau": 1.5, "lambda_": 0.0, "inverse_variance": 0}])
def test_score_fusion_bitwise_vs_oracle(pipeline, opts):
    """fuse_scored (crates/dense/src/fusion_score.rs:314-435) on the device against the restatement: candidates,
    adoption under mark_used and the (view, pixel) output order (image ids descend with the view index here, so key
    order would differ)."""
    wl, views, s = pipeline
    s.readout_resident(views, download=False)
    s.postprocess_resident(0, views)
    states = s.readout_download(0, views)
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src, image_ids=[1000 - v for v in range(len(wl.cams))])
    imgs = [scenes.unit_plane(kv.levels[0].pixels) for kv in wl.input.views]
    args = ([st.depth for st in states], [st.normal for st in states], [st.cost for st in states], imgs)
    prm = fusion.default_score_fusion(**opts)
    for vs in (views, views[1:]):
        n = s.fuse_scored_resident(0, vs, fc, prm)
        got = s.fused_points()
        want = oracle.fuse_scored(fc, *args, vs, prm)
        assert n == len(want) > 0
        np.testing.assert_array_equal(got.keys, want.keys)
        np.testing.assert_array_equal(got.positions, want.positions)
        np.testing.assert_array_equal(got.normals, want.normals)
        np.testing.assert_array_equal(got.colors, want.colors)
        np.testing.assert_array_equal(got.vis_counts, want.vis_counts)
        for i in range(len(want)):
            assert got.visibility(i) == want.visibility(i)


@pytest.mark.parametrize("smooth", [0, 2])
def test_score_fusion_with_visibility_and_smoothing_bitwise_vs_oracle(pipeline, smooth):
    """fuse_depth_maps_with(.., Some(score)) with its off-by-default steps on (crates/dense/src/densify.rs:535-556):
    the visibility filter over the adopted points, then `smooth` smoothing passes along normals, against the
    restatement of the same steps.  The filter must remove points and the smoothing must move some."""
    wl, views, s = pipeline
    s.readout_resident(views, download=False)
    s.postprocess_resident(0, views)
    states = s.readout_download(0, views)
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    imgs = [scenes.unit_plane(kv.levels[0].pixels) for kv in wl.input.views]
    args = ([st.depth for st in states], [st.normal for st in states], [st.cost for st in states], imgs)
    prm = fusion.default_score_fusion()
    post = fusion.default_fusion(2)
    post.visibility_check_views, post.visibility_min_violations, post.visibility_tau = 8, 1, 0.002
    post.smooth_iterations, post.smooth_radius_gsd = smooth, 2.0
    n = s.fuse_scored_resident(0, views, fc, prm, post=post)
    got = s.fused_points()
    want = oracle.fuse_scored(fc, *args, views, prm, post=post)
    assert n == len(want) > 0
    assert s.fused_visibility_removed == want.visibility_removed > 0
    np.testing.assert_array_equal(got.keys, want.keys)
    np.testing.assert_array_equal(got.positions, want.positions)
    np.testing.assert_array_equal(got.normals, want.normals)
    np.testing.assert_array_equal(got.vis_counts, want.vis_counts)
    if smooth:
        plain = fusion.default_fusion(2)
        plain.visibility_check_views, plain.visibility_min_violations, plain.visibility_tau = 8, 1, 0.002
        s.fuse_scored_resident(0, views, fc, prm, post=plain)
        assert (s.fused_points().positions != got.positions).any()  # the smoothing moved points


@pytest.mark.parametrize("residual", [0, 2])
def test_visibility_filter_bitwise_vs_oracle(pipeline, residual):
    """filter_visibility (crates/dense/src/visibility.rs:106-151) on the device cloud against the restatement: the
    kept points (both passes) and the removed count equal."""
    wl, views, s = pipeline
    s.readout_resident(views, download=False)
    s.postprocess_resident(0, views)
    states = s.readout_download(0, views)
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    imgs = [scenes.unit_plane(kv.levels[0].pixels) for kv in wl.input.views]
    prm = fusion.default_fusion(2)
    prm.residual = residual
    prm.visibility_check_views, prm.visibility_min_violations, prm.visibility_tau = 8, 1, 0.002
    n = s.fuse_resident(0, views, fc, prm)
    got = s.fused_points()
    want = oracle.fuse(fc, [st.depth for st in states], [st.normal for st in states], [st.cost for st in states],
                       imgs, views, prm)
    assert s.fused_visibility_removed == want.visibility_removed > 0
    assert n == len(want) and s.fused_residual == want.residual
    np.testing.assert_array_equal(got.keys, want.keys)
    np.testing.assert_array_equal(got.positions, want.positions)
    np.testing.assert_array_equal(got.normals, want.normals)
    np.testing.assert_array_equal(got.vis_counts, want.vis_counts)


@pytest.mark.parametrize("full", [False, True])
def test_smoothing_bitwise_vs_oracle(pipeline, full):
    """smooth_along_normals (crates/dense/src/smooth.rs:143-220) of the device cloud against the restatement (the
    same binary64 exponential on both sides): positions equal bit for bit; `full` adds the second pass and the
    visibility filter before it."""
    wl, views, s = pipeline
    s.readout_resident(views, download=False)
    s.postprocess_resident(0, views)
    states = s.readout_download(0, views)
    src = [list(kv.sources) for kv in wl.input.views]
    fc = fusion.FusionCams(wl.cams, src)
    imgs = [scenes.unit_plane(kv.levels[0].pixels) for kv in wl.input.views]
    prm = fusion.default_fusion(2)
    prm.smooth_iterations, prm.smooth_radius_gsd = 2, 2.0
    if full:
        prm.residual = 2
        prm.visibility_check_views, prm.visibility_min_violations, prm.visibility_tau = 8, 1, 0.002
    n = s.fuse_resident(0, views, fc, prm)
    got = s.fused_points()
    want = oracle.fuse(fc, [st.depth for st in states], [st.normal for st in states], [st.cost for st in states],
                       imgs, views, prm)
    assert n == len(want) > 0
    np.testing.assert_array_equal(got.keys, want.keys)
    np.testing.assert_array_equal(got.positions, want.positions)
    np.testing.assert_array_equal(got.normals, want.normals)
    prm.smooth_iterations = 0
    s.fuse_resident(0, views, fc, prm)
    assert (s.fused_points().positions != got.positions).any()  # the smoothing moved points


@pytest.mark.parametrize("full_k", [True, False])
def test_fill_holes_bitwise_vs_oracle(full_k):
    """Speckle removal then hole filling (fill_holes, crates/dense/src/postproc.rs:139-201) on the device readout,
    against the oracle on the same readout: planes, costs and counts equal bit for bit.  `full_k` passes the
    cameras' binary64 intrinsics; otherwise the levels' binary32 ones (the oracle gets the same values)."""
    wl = scenes.workload_small(160, 120, views=6, window_radius=3, seed=23, iters=2, sources=4, positions=2)
    views = list(range(len(wl.cams)))
    be = PatchMatchBackend(0, math="parity")
    with be.begin(wl.input) as s:
        s.schedule_resident(views, 2, 1, 1, graph=False)
        before = s.readout_resident(views)
        post = fusion.default_post()
        post.speckle_min_area_frac = 0.002
        post.fill_holes = 1
        post.fill_max_frac = 0.05
        ks = np.array([c.k for c in wl.cams], np.float64)
        if not full_k:
            ks = ks.astype(np.float32).astype(np.float64)
        removed, filled = s.postprocess_resident(0, views, post, intrinsics=ks if full_k else None, filled=True)
        got = s.readout_download(0, views)
    be.close()
    want_removed = want_filled = 0
    for v, (g, st) in enumerate(zip(got, before)):
        d, n, c = st.depth.copy(), st.normal.copy(), st.cost.copy()
        want_removed += oracle.remove_speckles(d, n, c, post)
        want_filled += oracle.fill_holes(d, n, c, st.cost, wl.input.views[v].levels[0].pixels, ks[v], post)
        np.testing.assert_array_equal(g.depth, d)
        np.testing.assert_array_equal(g.normal, n)
        np.testing.assert_array_equal(g.cost, c)
    assert (removed, filled) == (want_removed, want_filled)
    assert filled > 0
