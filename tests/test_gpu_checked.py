"""The bounds-checked build (ps_options.checked = 1, namespace ps_checked of the kernels).

Every data-dependent index of the half step, evaluate, filter, upsample, median, readout and snapshot kernels is
tested before its access; a failed test skips the access and records the first violation in a device fault word,
which the next synchronising call reports as PS_EFAULT.  Nothing traps and no test here makes an out-of-bounds
access: the checked kernels must give the parity build's bits (so they equal the CPU oracle) with the fault word
untouched, and the self-test probe (PS_INJECT_CHECK_PROBE) has the kernels test one index past the end of the state
arrays, which fails the test without any access and must surface as PS_EFAULT, after which the session runs on.
"""
import numpy as np
import pytest

from cumulus3d_b200 import _lib, densify, scenes
from cumulus3d_b200.patchstereo import DepthSnapshot, PatchMatchBackend, PsError, RunParams, ViewState
from oracle import oracle

pytestmark = pytest.mark.gpu


def _states(wl):
    return [ViewState.new(c.width, c.height) for c in wl.cams]


def _same(a, b, what):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.depth, y.depth, err_msg=what)
        np.testing.assert_array_equal(x.normal, y.normal, err_msg=what)
        np.testing.assert_array_equal(x.cost, y.cost, err_msg=what)


# two lanes per pixel; one lane + texture gather; row pairs + texture gather; staged source boxes + texture gather;
# row pairs + texture gather in the persistent kernel; staged boxes loaded by TMA + texture gather
@pytest.mark.parametrize("tuning", [0, 6, 10, 18, 42, 90])
def test_checked_kernels_equal_the_oracle(tuning):
    """Random init + photometric iterations, a geometric iteration through a snapshot, then the filter: the checked
    kernels report no violation and give the oracle's bits."""
    wl = scenes.workload_small(96, 72, views=3, window_radius=3, seed=31)
    p = RunParams(0, False, True, 3, 1)
    pg = RunParams(0, True, False, 1, 2)
    got = _states(wl)
    be = PatchMatchBackend(0, tuning=tuning, checked=True)
    assert "checked" in be.name()
    with be.begin(wl.input) as s:
        s.set_profiling(True)  # the staged path's counters
        s.run(wl.views, got, p)
        snap = DepthSnapshot(1, 0, [g.depth.copy() for g in got])
        s.run(wl.views, got, pg, snap)
        counts = s.filter(wl.views, got, snap)
        stats = s.kernel_stats(_lib.PS_KERNEL_HALF)
    be.close()
    ref = _states(wl)
    oracle.run(wl.input, wl.views, ref, p)
    oracle.run(wl.input, wl.views, ref, pg, snap)
    ccounts = oracle.filter(wl.input, wl.views, ref, snap)
    _same(got, ref, f"checked build, tuning {tuning}")
    for a, b in zip(counts, ccounts):
        np.testing.assert_array_equal(a, b)
    if tuning in (18, 90):
        assert stats["staged_windows"] > 0  # the staged path ran, so its box reads were tested


def test_checked_multiscale_schedule_equals_parity_build():
    """The on-device multi-scale schedule (upsample, median, readout and snapshot kernels included) under the checked
    build equals the parity build."""
    wl = scenes.workload_small(128, 96, views=3, window_radius=3, seed=17)
    views = []
    for v, cam in zip(wl.input.views, wl.cams):
        v.levels = densify.build_pyramid(v.levels[0].pixels, cam.k, 3)
        views.append(v)
    from cumulus3d_b200.patchstereo import KernelInput
    inp = KernelInput(views, 3, wl.input.pm, wl.input.filter, wl.input.seed)
    inp.filter.median_filter = 1
    sch = densify.Schedule(photometric_iters=2, photometric_iters_upper=1, geometric_rounds=1, geometric_iters=1)
    out = []
    for checked in (False, True):
        be = PatchMatchBackend(0, checked=checked)
        with be.begin(inp) as s:
            out.append(densify.compute_depth_maps_resident(s, inp, [0, 1, 2], sch))
        be.close()
    for a, b in zip(*out):
        np.testing.assert_array_equal(a.depth, b.depth)
        np.testing.assert_array_equal(a.normal, b.normal)


def test_probe_surfaces_as_efault_and_the_session_runs_on():
    wl = scenes.workload_small(80, 56, views=3, window_radius=3, seed=29)
    p = RunParams(0, False, True, 2, 1)
    be = PatchMatchBackend(0, checked=True)
    with be.begin(wl.input) as s:
        be.inject_failure(_lib.PS_INJECT_CHECK_PROBE)
        with pytest.raises(PsError) as e:
            s.run(wl.views, _states(wl), p)
        assert e.value.code == _lib.PS_EFAULT
        assert "self-test probe" in str(e.value)
        got = _states(wl)
        s.run(wl.views, got, p)  # the probe is spent and the fault word cleared
    be.close()
    ref = _states(wl)
    oracle.run(wl.input, wl.views, ref, p)
    _same(got, ref, "after the probe")


def test_probe_and_fast_math_need_a_checked_parity_backend():
    be = PatchMatchBackend(0)
    with pytest.raises(PsError) as e:
        be.inject_failure(_lib.PS_INJECT_CHECK_PROBE)
    assert e.value.code == _lib.PS_EINVAL
    be.close()
    with pytest.raises(PsError):
        PatchMatchBackend(0, math="fast", checked=True)
