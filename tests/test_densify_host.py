"""Host helpers of the driver (CPU only): pyramid, level count, readout threshold."""
import ctypes as C

import numpy as np

from cumulus3d_b200 import densify
from cumulus3d_b200.patchstereo import ViewState
from oracle import oracle


def test_num_levels_reference_values():
    assert densify.num_levels(539, 3, 64) == 3
    assert densify.num_levels(240, 3, 64) == 2
    assert densify.num_levels(90, 3, 64) == 1


def test_pyramid_matches_oracle_restatement():
    rng = np.random.default_rng(3)
    g = rng.integers(0, 256, (37, 53), dtype=np.uint8)
    k = (50.0, 51.0, 26.0, 18.0)
    pyr = densify.build_pyramid(g, k, 3)
    assert [lv.pixels.shape for lv in pyr] == [(9, 13), (18, 26), (37, 53)]
    cur, kk = g, k
    for lvl in (1, 0):
        h, w = cur.shape
        out = np.zeros((h // 2, w // 2), np.uint8)
        ko = (C.c_double * 4)()
        oracle.lib().oracle_pyramid_step(np.ascontiguousarray(cur).ctypes.data, w, h, (C.c_double * 4)(*kk),
                                         out.ctypes.data, ko)
        assert np.array_equal(out, pyr[lvl].pixels)
        assert np.allclose(list(ko), pyr[lvl].k, rtol=0, atol=1e-12)
        cur, kk = out, tuple(ko)


def test_pyramid_intrinsics_reference_case():
    p = densify.build_pyramid(np.full((7, 9), 100, np.uint8), (10.0, 10.0, 4.0, 3.0), 2)
    assert (p[0].width, p[0].height, p[1].width) == (4, 3, 9)
    assert abs(p[0].k[2] - 1.75) < 1e-6 and abs(p[0].k[0] - 5.0) < 1e-6
    assert (p[0].pixels == 100).all()


def test_readout_threshold():
    s = ViewState.new(4, 1)
    s.depth[...] = [1.0, 2.0, 0.0, 3.0]
    s.normal[...] = [0.0, 0.0, -1.0]
    counts = np.array([[0, 2, 5, 3]], np.uint8)
    out = densify.readout([s], [counts], [4], 3)[0]
    assert out.depth.tolist() == [[0.0, 0.0, 0.0, 3.0]]
    assert (out.normal[0, 3] == [0, 0, -1]).all() and (out.normal[0, 0] == 0).all()
    # fewer sources than min_num_consistent: need = nsrc (and at least 1)
    out = densify.readout([s], [counts], [2], 3)[0]
    assert out.depth.tolist() == [[0.0, 2.0, 0.0, 3.0]]
