"""Properties of the CPU oracle on seeded synthetic scenes (CPU only, small sizes)."""
import numpy as np
import pytest

from cumulus3d_b200 import scenes
from cumulus3d_b200.patchstereo import DepthSnapshot, RunParams, ViewState
from oracle import oracle


@pytest.fixture(scope="module")
def small():
    return scenes.workload_small(120, 90, window_radius=3, seed=31)


def test_thread_count_does_not_change_bits(small):
    """Red-black updates read only the other colour, so the result is independent of the thread schedule."""
    p = RunParams(0, False, True, 2, 1)
    a = [ViewState.new(c.width, c.height) for c in small.cams]
    b = [ViewState.new(c.width, c.height) for c in small.cams]
    oracle.run(small.input, small.views, a, p, threads=1)
    oracle.run(small.input, small.views, b, p, threads=8)
    for x, y in zip(a, b):
        assert np.array_equal(x.depth, y.depth) and np.array_equal(x.normal, y.normal)
        assert np.array_equal(x.cost, y.cost)


def test_reference_acceptance_gate():
    """The reference's own acceptance gate (crates/cuda/tests/patchmatch_gpu.rs:96-98 and :118-132) on its own
    synthetic scene (crates/dense/src/synthetic.rs, restated in csrc/ps_synth.cpp), run by the oracle through the whole
    fast-profile flow: median depth error < 0.005, median normal error < 3°, valid > 0.5, and a fused cloud of more
    than 10 000 points on the scene's surfaces."""
    import reference_gate as rg
    g = rg.setup(oracle.select_neighbors)
    assert g.input.num_levels == 3 and all(len(s) == 8 for s in g.sources)
    depths, normals, _, cloud = rg.run_oracle(g)
    rg.check(rg.accuracy(g.scene, depths, normals), rg.fusion_stats(g.scene, cloud.positions))


def test_converges_to_ground_truth(small):
    """A raw single-level run (no filter, no post-processing, 2 sources) on a terrain scene converges toward the ground
    truth on the centre view; the reference's own thresholds apply to its full flow (test_reference_acceptance_gate)."""
    st = [ViewState.new(c.width, c.height) for c in small.cams]
    oracle.run(small.input, small.views, st, RunParams(0, False, True, 4, 1))
    gt, gn = small.gt_depth[1], small.gt_normal[1]
    s = st[1]
    m = (gt > 0) & (s.depth > 0)
    assert m.mean() > 0.5
    relerr = np.abs(s.depth[m] - gt[m]) / gt[m]
    assert np.median(relerr) < 0.005
    ang = np.degrees(np.arccos(np.clip((s.normal * gn).sum(-1)[m], -1, 1)))
    assert np.median(ang) < 8.0


def test_filter_on_ground_truth_counts_sources(small):
    """Ground-truth planes pass the geometric filter against ground-truth snapshots for most pixels."""
    st = []
    for i, c in enumerate(small.cams):
        s = ViewState.new(c.width, c.height)
        s.depth[...] = small.gt_depth[i]
        s.normal[...] = small.gt_normal[i]
        st.append(s)
    snap = DepthSnapshot(1, 0, [g.copy() for g in small.gt_depth])
    counts = oracle.filter(small.input, small.views, st, snap)
    assert (counts[1] >= 1).mean() > 0.6


def _tilted_plane_level_pair():
    hk = (40.0, 40.0, 15.5, 11.5)
    lk = (20.0, 20.0, (15.5 + 0.5) * 0.5 - 0.5, (11.5 + 0.5) * 0.5 - 0.5)
    v = np.array([0.3, -0.2, -1.0])
    n = v / np.linalg.norm(v)

    def ray(k, x, y):
        return np.array([(x - k[2]) / k[0], (y - k[3]) / k[1], 1.0])

    def hit(r):
        return -5.0 / n.dot(r)
    return hk, lk, n, ray, hit


def test_upsample_reproduces_plane_and_median_keeps_it():
    """crates/dense/src/upsample.rs:278-307 through the oracle's restatement of pm_upsample / pm_median."""
    from cumulus3d_b200.patchstereo import KernelInput, KernelView, LevelImage
    hk, lk, n, ray, hit = _tilted_plane_level_pair()
    lo = LevelImage(np.full((12, 16), 50, np.uint8), lk)
    hi = LevelImage(np.full((24, 32), 50, np.uint8), hk)
    inp = KernelInput([KernelView(1, [lo, hi], [], [], 1.0, 100.0)], 2)
    low = ViewState.new(16, 12)
    for y in range(12):
        for x in range(16):
            low.depth[y, x] = hit(ray(lk, x, y))
            low.normal[y, x] = n
    up = oracle.upsample(inp, 1, [0], [low], 1.0, 0.04)[0]
    t = np.array([[hit(ray(hk, x, y)) for x in range(32)] for y in range(24)])
    assert np.max(np.abs(up.depth - t) / t) < 1e-5
    md = oracle.median(inp, 1, [0], [up])[0]
    assert abs(md.depth.ravel()[100] - up.depth.ravel()[100]) / up.depth.ravel()[100] < 1e-5


def test_fp64_reevaluation_close_to_fp32(small):
    """The FP64 re-evaluation of converged hypotheses agrees with the fp32 top-K cost to ~1e-5."""
    st = [ViewState.new(c.width, c.height) for c in small.cams]
    oracle.run(small.input, small.views, st, RunParams(0, False, True, 2, 1))
    c32 = oracle.evaluate(small.input, 0, [1], [st[1]])[0]
    c64 = oracle.reeval_f64(small.input, 0, [1], [st[1]])[0]
    ok = (c32 < 1.5) & (c64 < 1.5)
    assert ok.mean() > 0.5
    assert np.median(np.abs(c32[ok] - c64[ok])) < 1e-5


@pytest.mark.parametrize("case", ["radius20", "sources32"])
def test_oracle_runs_at_the_abi_limits(case):
    """The limits the reference validates (crates/cuda/src/patchmatch.rs:292-294, :366-371): window radius 20 (a
    41×41 window larger than the image) and 32 sources.  The restatement runs there, with finite costs in [0, 2]
    positive depths and unit normals."""
    if case == "radius20":
        wl = scenes.workload_small(32, 24, views=3, window_radius=20, seed=5, sources=2)
    else:
        wl = scenes.workload_small(24, 16, views=33, window_radius=1, seed=6, sources=32, positions=11)
        assert all(len(kv.sources) == 32 for kv in wl.input.views)
    st = [ViewState.new(c.width, c.height) for c in wl.cams]
    oracle.run(wl.input, wl.views, st, RunParams(0, False, True, 1, 1))
    for s in st:
        assert np.isfinite(s.cost).all() and (s.cost >= 0).all() and (s.cost <= 2).all()
        assert np.isfinite(s.depth).all() and (s.depth > 0).all()
        assert np.allclose(np.linalg.norm(s.normal, axis=-1), 1.0, atol=1e-4)
