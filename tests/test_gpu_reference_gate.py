"""The reference's acceptance gate on the engine (crates/cuda/tests/patchmatch_gpu.rs:96-98, :118-132): its synthetic
scene densified through the whole fast-profile flow on the GPU (neighbour selection, the multi-scale schedule in one
graph, readout, speckle removal, hole filling, consistency fusion) meets the reference's thresholds, and every stage's
result equals the CPU oracle's bit for bit."""
import numpy as np
import pytest

import reference_gate as rg
from cumulus3d_b200 import neighbors
from cumulus3d_b200.patchstereo import PatchMatchBackend
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_reference_gate_on_engine_equals_oracle():
    g = rg.setup(neighbors.select_neighbors)
    want = oracle.select_neighbors(g.scene.model, rg.NeighborParams())
    assert g.sources == want.sources and g.input.num_levels == 3
    be = PatchMatchBackend(0, math="parity")
    with be.begin(g.input) as s:
        depths, normals, costs, cloud = rg.run_engine(g, s)
    be.close()
    acc = rg.accuracy(g.scene, depths, normals)
    fus = rg.fusion_stats(g.scene, cloud.positions)
    rg.check(acc, fus)
    od, on, oc, ocloud = rg.run_oracle(g)
    for v in range(len(depths)):
        np.testing.assert_array_equal(depths[v], od[v], err_msg=f"depth view {v}")
        np.testing.assert_array_equal(normals[v], on[v], err_msg=f"normal view {v}")
        np.testing.assert_array_equal(costs[v], oc[v], err_msg=f"cost view {v}")
    np.testing.assert_array_equal(cloud.keys, ocloud.keys)
    np.testing.assert_array_equal(cloud.positions, ocloud.positions)
