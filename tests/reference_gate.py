"""The reference's own acceptance gate for PatchStereo, restated: its synthetic scene (crates/dense/src/synthetic.rs,
make_scene with SynthConfig::default(): 9 views of 384×288, f = 300, a 3×3 grid at 20 m over a textured floor with two
boxes), densified with the fast profile (crates/dense/src/params.rs:440-503: window radius 5 step 2, 3 scales, 6 + 3
photometric iterations, 2 geometric rounds of 2, the tuned filter, speckle removal and hole filling), scored as
crates/cuda/tests/patchmatch_gpu.rs:46-73 scores it (median relative depth error, median normal error and valid
fraction of the final maps against the ground truth) and its consistency fusion checked against the scene's surfaces
(:118-132).  The thresholds are the reference's: depth < 0.005, normals < 3°, valid > 0.5; more than 10 000 fused
points, median surface distance < 0.02 m, under 2 % beyond 0.1 m.

Shared by the CPU test (the oracle runs the whole flow) and the GPU test (the engine runs it, and must also equal the
oracle bit for bit).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from cumulus3d_b200 import densify, fusion, scenes
from cumulus3d_b200.neighbors import NeighborParams

DEPTH_MEDIAN_MAX = 0.005
NORMAL_MEDIAN_MAX_DEG = 3.0
VALID_MIN = 0.5
FUSED_MIN = 10_000
SURFACE_MEDIAN_MAX = 0.02  # and fewer than 1 in 50 points beyond 0.1 m


@dataclass
class Gate:
    scene: scenes.ReferenceScene
    input: object
    sources: List[List[int]]
    overlap: List[List[int]]


def setup(select) -> Gate:
    """The scene, its neighbours and depth ranges (`select` = ps_select_neighbors or its CPU restatement, default
    NeighborParams: 10 sources, 1°, plain selection) and the fast-profile input."""
    sc = scenes.reference_scene()
    nb = select(sc.model, NeighborParams(), pair_stats=True)
    inp = densify.kernel_input(sc.cams, sc.gray, nb.sources, nb.depth_ranges)
    lim = int(fusion.default_fusion().consistency_num_images)
    n = len(sc.cams)
    cnt = nb.pair_count
    overlap = []
    for v in range(n):  # PairStats::select(v, lim, 0.0): descending shared count, ascending index
        c = [(-int(cnt[min(v, o), max(v, o)]), o) for o in range(n) if o != v and cnt[min(v, o), max(v, o)] > 0]
        overlap.append([o for _, o in sorted(c)[:lim]])
    return Gate(sc, inp, nb.sources, overlap)


def post_params():
    """PostParams::default() with the fast profile's hole filling (params.rs:452-459)."""
    p = fusion.default_post()
    p.fill_holes = 1
    return p


def fusion_params():
    """FusionParams with the fast profile's tuning (params.rs:456-459): 3 views, 0.5 % depth, 23°, 100 px."""
    p = fusion.default_fusion()
    p.min_consistent_views, p.max_depth_error, p.max_normal_error_deg, p.max_reproj_error = 3, 0.005, 23.0, 100.0
    return p


def fusion_cams(g: Gate):
    return fusion.FusionCams(g.scene.cams, g.sources, overlap=g.overlap, image_ids=g.scene.image_ids)


def accuracy(sc: scenes.ReferenceScene, depths: Sequence[np.ndarray], normals: Sequence[np.ndarray]) -> dict:
    """patchmatch_gpu.rs:46-73: over every pixel of every view, the pixels where both the map and the ground truth
    have depth > 0 count as valid; relative depth error and the normal angle (dot product in binary32, acos in
    binary64) of those; medians are the upper middle element."""
    de, ne = [], []
    total = 0
    for v, (d, n) in enumerate(zip(depths, normals)):
        t = sc.gt_depth[v]
        total += d.size
        ok = (d > 0) & (t > 0)
        de.append(np.abs(d[ok].astype(np.float64) - t[ok]) / t[ok])
        a = n.reshape(d.shape + (3,))[ok]
        b = sc.gt_normal[v][ok]
        c = (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]).astype(np.float64)
        ne.append(np.degrees(np.arccos(np.clip(c, -1.0, 1.0))))
    de = np.sort(np.concatenate(de))
    ne = np.sort(np.concatenate(ne))
    return {"valid": len(de) / total, "depth_median": float(de[len(de) // 2]),
            "depth_p90": float(de[len(de) * 9 // 10]), "normal_median_deg": float(ne[len(ne) // 2])}


def fusion_stats(sc: scenes.ReferenceScene, positions: np.ndarray) -> dict:
    """patchmatch_gpu.rs:118-132: point count, median distance to the scene's surfaces, points beyond 0.1 m."""
    d = sc.surface_distances(positions)
    n = len(d)
    return {"points": n, "surface_median": float(np.sort(d)[n // 2]) if n else float("inf"),
            "far": int((d > 0.1).sum())}


def check(acc: dict, fus: dict) -> None:
    assert acc["depth_median"] < DEPTH_MEDIAN_MAX, acc
    assert acc["normal_median_deg"] < NORMAL_MEDIAN_MAX_DEG, acc
    assert acc["valid"] > VALID_MIN, acc
    assert fus["points"] > FUSED_MIN, fus
    assert fus["surface_median"] < SURFACE_MEDIAN_MAX, fus
    assert fus["far"] * 50 < fus["points"], fus


def run_oracle(g: Gate, threads=None):
    """The whole flow on the CPU restatement: compute_depth_maps (host driver over OracleSession), readout, speckle
    removal and hole filling per view, consistency fusion.  Returns (depths, normals, costs, cloud)."""
    from oracle import oracle
    views = list(range(len(g.scene.cams)))
    sess = oracle.OracleSession(g.input, threads)
    _, filtered, _ = densify.compute_depth_maps(sess, g.input, views)
    post = post_params()
    depths, normals, costs = [], [], []
    for v, st in zip(views, filtered):
        d = np.ascontiguousarray(st.depth, np.float32).copy()
        n = np.ascontiguousarray(st.normal, np.float32).reshape(d.shape + (3,)).copy()
        c = np.ascontiguousarray(st.cost, np.float32).copy()
        oracle.remove_speckles(d, n, c, post)
        oracle.fill_holes(d, n, c, st.cost, g.scene.gray[v], g.scene.cams[v].k, post)
        depths.append(d)
        normals.append(n)
        costs.append(c)
    cloud = oracle.fuse(fusion_cams(g), depths, normals, costs,
                        [scenes.unit_plane(g.scene.gray[v]) for v in views], views, fusion_params(), threads)
    return depths, normals, costs, cloud


def run_engine(g: Gate, session):
    """The whole flow on the device: the multi-scale schedule in one graph (ps_schedule_multiscale), post-processing
    of the resident readout (speckles, hole filling), consistency fusion.  Returns (depths, normals, costs, cloud)."""
    views = list(range(len(g.scene.cams)))
    top = g.input.num_levels - 1
    densify.compute_depth_maps_resident(session, g.input, views)
    session.postprocess_resident(top, views, post_params(), intrinsics=np.array([c.k for c in g.scene.cams]))
    final = session.readout_download(top, views)
    session.fuse_resident(top, views, fusion_cams(g), fusion_params())
    cloud = session.fused_points()
    return ([s.depth for s in final], [s.normal.reshape(s.depth.shape + (3,)) for s in final],
            [s.cost for s in final], cloud)
