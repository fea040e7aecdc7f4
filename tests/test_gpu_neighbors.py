"""Neighbour views and depth ranges on the GPU (ps_select_neighbors) against the CPU oracle: the reference's
known-answer scene, seeded random models (repeated views in tracks, unobserved views, empty models) in plain and
direction-diverse modes, and sparse tracks of a rendered scene.  Counts, selections and depth ranges must be equal;
the 75th-percentile angles go through CUDA's acos on the device and the platform's on the CPU, so they are compared
to 1e-6 relative (both round each angle to binary32 first)."""
import numpy as np
import pytest

from cumulus3d_b200 import scenes
from cumulus3d_b200.neighbors import NeighborParams, SparseModel, select_neighbors
from oracle import oracle
from test_neighbors_oracle import known_answer_model, random_model

pytestmark = pytest.mark.gpu


def _same(m: SparseModel, p: NeighborParams):
    g = select_neighbors(m, p, pair_stats=True)
    c = oracle.select_neighbors(m, p, pair_stats=True)
    assert g.sources == c.sources
    assert g.depth_ranges == c.depth_ranges
    n = m.num_views
    upper = np.triu(np.ones((n, n), bool), 1)
    np.testing.assert_array_equal(g.pair_count[upper], c.pair_count[upper])
    np.testing.assert_allclose(g.pair_angle75[upper], c.pair_angle75[upper], rtol=1e-6, atol=0)
    return g


def test_known_answer_scene():
    m = known_answer_model()
    assert _same(m, NeighborParams(10, 1.0)).sources[0] == [1, 3]
    assert _same(m, NeighborParams(10, 0.0)).sources[0] == [2, 1, 3]


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("params", [NeighborParams(4, 1.0), NeighborParams(10, 0.0), NeighborParams(3, 5.0),
                                    NeighborParams(4, 1.0, 8, 0.5), NeighborParams(6, 0.0, 4, 0.25)])
def test_random_models(seed, params):
    _same(random_model(seed, nv=11, npts=3000, max_track=8), params)


def test_empty_model():
    m = known_answer_model()
    empty = SparseModel(m.views, np.zeros((0, 3)), np.zeros(1, np.uint32), np.zeros(0, np.uint32))
    g = _same(empty, NeighborParams())
    assert all(s == [] for s in g.sources) and all(r is None for r in g.depth_ranges)


@pytest.mark.parametrize("params", [NeighborParams(2, 1.0), NeighborParams(2, 0.0, 8, 0.5)])
def test_rendered_scene_tracks(params):
    wl = scenes.workload_c1(seed=1)
    m = scenes.sparse_model(wl.cams, wl.gt_depth, 6000, seed=3)
    g = _same(m, params)
    assert all(len(s) == 2 for s in g.sources)
