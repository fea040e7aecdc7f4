"""The multi-scale driver (compute_depth_maps schedule) on the engine equals the same schedule on the oracle."""
import numpy as np
import pytest

from cumulus3d_b200 import densify, scenes
from cumulus3d_b200.patchstereo import KernelInput
from oracle.oracle import OracleSession

pytestmark = pytest.mark.gpu


def _pyramid_input(wl, levels=3, weak_var=0.0, median=True):
    views = []
    for v, cam in zip(wl.input.views, wl.cams):
        px = v.levels[0].pixels  # 8-bit gray, as the reference takes it
        g = px if px.dtype == np.uint8 else scenes.to_gray8(px)
        v.levels = densify.build_pyramid(g, cam.k, levels)
        views.append(v)
    inp = KernelInput(views, levels, wl.input.pm, wl.input.filter, wl.input.seed)
    inp.pm.weak_texture_var = weak_var
    inp.filter.median_filter = int(median)
    return inp


@pytest.mark.parametrize("weak_var", [0.0, 0.002])
def test_multiscale_schedule_bitwise_equal(backend, weak_var):
    wl = scenes.workload_small(128, 96, views=3, window_radius=3, seed=17)
    inp = _pyramid_input(wl, 3, weak_var)
    sch = densify.Schedule(photometric_iters=2, photometric_iters_upper=1, geometric_rounds=1, geometric_iters=1)
    with backend.begin(inp) as s:
        g_raw, g_fin, g_cnt = densify.compute_depth_maps(s, inp, [0, 1, 2], sch, weak_texture_prior=weak_var > 0)
    c_raw, c_fin, c_cnt = densify.compute_depth_maps(OracleSession(inp), inp, [0, 1, 2], sch,
                                                     weak_texture_prior=weak_var > 0)
    for a, b in zip(g_raw, c_raw):
        np.testing.assert_array_equal(a.depth, b.depth)
        np.testing.assert_array_equal(a.normal, b.normal)
    for a, b in zip(g_cnt, c_cnt):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(g_fin, c_fin):
        np.testing.assert_array_equal(a.depth, b.depth)
    assert sum(float((f.depth > 0).mean()) for f in g_fin) > 0.3


@pytest.mark.parametrize("weak_var,graph", [(0.0, True), (0.0, False), (0.002, True)])
def test_multiscale_on_device_equals_host_driver(backend, weak_var, graph):
    """ps_schedule_multiscale (every level on the device, one graph launch) = the host-driven compute_depth_maps."""
    wl = scenes.workload_small(128, 96, views=3, window_radius=3, seed=17)
    inp = _pyramid_input(wl, 3, weak_var)
    sch = densify.Schedule(photometric_iters=2, photometric_iters_upper=1, geometric_rounds=1, geometric_iters=1)
    with backend.begin(inp) as s:
        _, h_fin, _ = densify.compute_depth_maps(s, inp, [0, 1, 2], sch, weak_texture_prior=weak_var > 0)
    with backend.begin(inp) as s:
        d_fin = densify.compute_depth_maps_resident(s, inp, [0, 1, 2], sch, weak_texture_prior=weak_var > 0,
                                                    graph=graph)
        again = densify.compute_depth_maps_resident(s, inp, [0, 1, 2], sch, weak_texture_prior=weak_var > 0,
                                                    graph=graph)  # a replay gives the same maps
    for a, b, c in zip(d_fin, h_fin, again):
        np.testing.assert_array_equal(a.depth, b.depth)
        np.testing.assert_array_equal(a.normal, b.normal)
        np.testing.assert_array_equal(a.depth, c.depth)


@pytest.mark.parametrize("shape,levels", [((96, 128), 3), ((1080, 1920), 4), ((77, 131), 3)])
def test_pyramid_on_device_equals_host(shape, levels):
    """ps_build_pyramid (GPU) = build_pyramid (host restatement of upsample.rs:46-102), levels and intrinsics."""
    rng = np.random.default_rng(shape[0])
    gray = rng.integers(0, 256, shape, dtype=np.uint8)
    k = (1663.0, 1663.5, (shape[1] - 1) / 2.0, (shape[0] - 1) / 2.0)
    host = densify.build_pyramid(gray, k, levels)
    dev = densify.build_pyramid_device(gray, k, levels)
    assert len(host) == len(dev) == levels
    for a, b in zip(host, dev):
        np.testing.assert_array_equal(a.pixels, b.pixels)
        assert tuple(a.k) == tuple(b.k)
