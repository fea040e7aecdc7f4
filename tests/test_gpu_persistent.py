"""The persistent half step (PS_TUNE_PERSISTENT): every half step of a run in one launch over a device work queue of
(half step, tile) items, with bounded per-view waits between half steps.

* the results are the per-launch kernels' bits (so the CPU oracle's), for single runs, ragged batches of mixed
  sizes, geometric runs and the captured single-level schedule;
* a run is one half-step launch instead of two per iteration;
* the stall switch (PS_INJECT_QUEUE_STALL) makes the waits need one tile more than exists: the first wait runs out
  its bounded spin, the call fails with PS_ETIMEOUT, and the session runs on (nothing hangs and nothing faults).
"""
import time

import numpy as np
import pytest

from cumulus3d_b200 import _lib, scenes
from cumulus3d_b200.patchstereo import DepthSnapshot, PatchMatchBackend, PsError, RunParams, ViewState
from oracle import oracle

pytestmark = pytest.mark.gpu

ROW_PAIRS_TEX = _lib.PS_TUNE_ROW_PAIRS | _lib.PS_TUNE_TEX_GATHER
PERSISTENT = ROW_PAIRS_TEX | _lib.PS_TUNE_PERSISTENT


def _states(wl):
    return [ViewState.new(c.width, c.height) for c in wl.cams]


def _same(a, b, what):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.depth, y.depth, err_msg=what)
        np.testing.assert_array_equal(x.normal, y.normal, err_msg=what)
        np.testing.assert_array_equal(x.cost, y.cost, err_msg=what)


@pytest.mark.parametrize("tuning", [PERSISTENT, PERSISTENT & ~_lib.PS_TUNE_TEX_GATHER])
def test_persistent_runs_equal_the_oracle(tuning):
    wl = scenes.workload_small(112, 80, views=3, window_radius=3, seed=41)
    p = RunParams(0, False, True, 3, 1)
    pg = RunParams(0, True, False, 2, 2)
    got = _states(wl)
    be = PatchMatchBackend(0, tuning=tuning)
    with be.begin(wl.input) as s:
        s.set_profiling(True)
        s.run(wl.views, got, p)
        snap = DepthSnapshot(1, 0, [g.depth.copy() for g in got])
        s.run(wl.views, got, pg, snap)
        half = s.kernel_stats(_lib.PS_KERNEL_HALF)
    be.close()
    assert half["launches"] == 2  # one persistent launch per run (3 + 2 iterations, 10 half steps)
    ref = _states(wl)
    oracle.run(wl.input, wl.views, ref, p)
    oracle.run(wl.input, wl.views, ref, pg, snap)
    _same(got, ref, f"persistent, tuning {tuning:#x}")


def test_persistent_ragged_batch_equals_per_launch_kernels():
    """Views of three sizes in one batch (different tile counts per view, so the per-view waits count different
    totals): persistent = one launch per half step, bit for bit, through the resident schedule and its graph."""
    parts = [scenes.workload_small(w, h, views=2, window_radius=3, seed=50 + i)
             for i, (w, h) in enumerate([(64, 48), (150, 70), (96, 120)])]
    inp = parts[0].input
    for extra in parts[1:]:
        off = len(inp.views)
        for v in extra.input.views:
            v.sources = [j + off for j in v.sources]
            inp.views.append(v)
    views = list(range(len(inp.views)))
    out = []
    for tuning in (ROW_PAIRS_TEX, PERSISTENT):
        be = PatchMatchBackend(0, tuning=tuning)
        with be.begin(inp) as s:
            s.schedule_resident(views, 3, 1, 1, graph=True)
            s.schedule_resident(views, 3, 1, 1, graph=True)  # a replay of the captured graph
            out.append(s.readout_download(0, views))
        be.close()
    _same(out[0], out[1], "persistent vs per-launch, ragged batch")


def test_queue_stall_times_out_and_the_session_runs_on():
    wl = scenes.workload_small(96, 64, views=3, window_radius=3, seed=43)
    p = RunParams(0, False, True, 2, 1)
    be = PatchMatchBackend(0, tuning=PERSISTENT)
    with be.begin(wl.input) as s:
        be.inject_failure(_lib.PS_INJECT_QUEUE_STALL)
        t0 = time.time()
        with pytest.raises(PsError) as e:
            s.run(wl.views, _states(wl), p)
        assert e.value.code == _lib.PS_ETIMEOUT
        assert time.time() - t0 < 60.0
        got = _states(wl)
        s.run(wl.views, got, p)  # the stall is spent and the error word cleared
    be.close()
    ref = _states(wl)
    oracle.run(wl.input, wl.views, ref, p)
    _same(got, ref, "after the queue stall")
