"""Failure handling of the engine, made on the host (no GPU fault, trap or hang): status codes of the reference's error
mapping (crates/cuda/src/patchmatch.rs:234-236, :258, :292-294, :641) and a backend that stays usable afterwards.

* a second session on a busy backend: PS_EBUSY (the reference's backend holds a mutex for the session's life);
* an injected device-allocation failure: PS_ENOMEM from ps_begin; an injected upload failure: PS_ECUDA from ps_begin
  and from ps_run; each time the next session or call runs normally and equals the CPU oracle bit for bit;
* malformed states (NaN, infinite and negative depths, NaN normals) run to completion with the oracle's bits;
* a snapshot map of the wrong size is left out, as the reference leaves it out, and a snapshot of another level is
  rejected with PS_EINVAL.
"""
import numpy as np
import pytest

from cumulus3d_b200 import _lib, scenes
from cumulus3d_b200.patchstereo import DepthSnapshot, PatchMatchBackend, PsError, RunParams, ViewState
from oracle import oracle

pytestmark = pytest.mark.gpu


def _wl():
    return scenes.workload_small(80, 56, views=3, window_radius=3, seed=29)


def _states(wl):
    return [ViewState.new(c.width, c.height) for c in wl.cams]


def _same(a, b, what):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.depth, y.depth, err_msg=what)
        np.testing.assert_array_equal(x.normal, y.normal, err_msg=what)
        np.testing.assert_array_equal(x.cost, y.cost, err_msg=what)


def _oracle_run(wl, p, states=None, snap=None):
    st = states if states is not None else _states(wl)
    oracle.run(wl.input, wl.views, st, p, snap)
    return st


def test_second_session_on_a_busy_backend():
    wl = _wl()
    be = PatchMatchBackend(0)
    s = be.begin(wl.input)
    with pytest.raises(PsError) as e:
        be.begin(wl.input)
    assert e.value.code == _lib.PS_EBUSY
    s.close()
    p = RunParams(0, False, True, 2, 1)
    got = _states(wl)
    with be.begin(wl.input) as s2:
        s2.run(wl.views, got, p)
    be.close()
    _same(got, _oracle_run(wl, p), "after PS_EBUSY")


@pytest.mark.parametrize("after", [0, 3, 9])
def test_injected_device_allocation_failure(after):
    """The (after+1)-th device allocation of ps_begin fails: PS_ENOMEM, the partial session is torn down, and the
    next session on the same backend runs normally."""
    wl = _wl()
    be = PatchMatchBackend(0)
    be.inject_failure(_lib.PS_INJECT_DEVICE_ALLOC, after)
    with pytest.raises(PsError) as e:
        be.begin(wl.input)
    assert e.value.code == _lib.PS_ENOMEM
    p = RunParams(0, False, True, 2, 1)
    got = _states(wl)
    with be.begin(wl.input) as s:
        s.run(wl.views, got, p)
    be.close()
    _same(got, _oracle_run(wl, p), f"after an allocation failure ({after})")


def test_injected_upload_failures():
    """An image upload failing in ps_begin and a state upload failing in ps_run: PS_ECUDA both times; the session of
    the second case stays usable, and the rerun equals the oracle."""
    wl = _wl()
    be = PatchMatchBackend(0)
    be.inject_failure(_lib.PS_INJECT_UPLOAD, 0)
    with pytest.raises(PsError) as e:
        be.begin(wl.input)
    assert e.value.code == _lib.PS_ECUDA
    p = RunParams(0, False, True, 2, 1)
    cont = RunParams(0, False, False, 1, 2)  # continues from the caller's states: they are uploaded
    with be.begin(wl.input) as s:
        got = _states(wl)
        s.run(wl.views, got, p)
        start = [g.copy() for g in got]
        be.inject_failure(_lib.PS_INJECT_UPLOAD, 0)
        with pytest.raises(PsError) as e2:
            s.run(wl.views, [g.copy() for g in start], cont)
        assert e2.value.code == _lib.PS_ECUDA
        s.run(wl.views, got, cont)
    be.close()
    want = _oracle_run(wl, p)
    oracle.run(wl.input, wl.views, want, cont)
    _same(got, want, "after an upload failure")


def test_malformed_states_run_like_the_oracle():
    """Continuing from states with NaN, infinite, zero and negative depths and NaN normals: the run completes and its
    result equals the oracle's (both treat such planes as invalid hypotheses; the refinement replaces them)."""
    wl = _wl()
    rng = np.random.default_rng(5)
    base = _states(wl)
    for st in base:
        st.depth[...] = rng.uniform(25.0, 60.0, st.depth.shape).astype(np.float32)
        n = rng.normal(0.0, 0.2, st.normal.shape).astype(np.float32) + np.float32([0.0, 0.0, -1.0])
        st.normal[...] = n / np.linalg.norm(n, axis=-1, keepdims=True)
        st.cost[...] = 1.0
        bad = rng.random(st.depth.shape)
        st.depth[bad < 0.05] = np.nan
        st.depth[(bad >= 0.05) & (bad < 0.08)] = np.inf
        st.depth[(bad >= 0.08) & (bad < 0.12)] = -5.0
        st.depth[(bad >= 0.12) & (bad < 0.14)] = 0.0
        st.normal[(bad >= 0.14) & (bad < 0.17)] = np.nan
    p = RunParams(0, False, False, 2, 1)
    be = PatchMatchBackend(0)
    got = [s.copy() for s in base]
    with be.begin(wl.input) as s:
        s.run(wl.views, got, p)
    be.close()
    _same(got, _oracle_run(wl, p, [s.copy() for s in base]), "malformed states")
    assert all(np.isfinite(g.cost).all() for g in got)


def test_snapshot_of_wrong_size_or_level():
    wl = _wl()
    p1 = RunParams(0, False, True, 2, 1)
    be = PatchMatchBackend(0)
    with be.begin(wl.input) as s:
        got = _states(wl)
        s.run(wl.views, got, p1)
        ref = [g.copy() for g in got]
        # view 1's map has the wrong length: left out, exactly as if it were missing
        maps = [g.depth.copy() for g in got]
        maps[1] = maps[1].ravel()[:-7]
        p2 = RunParams(0, True, False, 1, 2)
        s.run(wl.views, got, p2, DepthSnapshot(7, 0, maps))
        missing = [m if v != 1 else None for v, m in enumerate([g.depth.copy() for g in ref])]
        alt = [r.copy() for r in ref]
        s.run(wl.views, alt, p2, DepthSnapshot(8, 0, missing))
        _same(got, alt, "wrong-size map = missing map")
        want = [r.copy() for r in ref]
        oracle.run(wl.input, wl.views, want, p2, DepthSnapshot(7, 0, maps))
        _same(got, want, "wrong-size map, oracle")
        # a snapshot of a level the session does not have
        with pytest.raises(PsError) as e:
            s.run(wl.views, [r.copy() for r in ref], p2, DepthSnapshot(9, 3, [r.depth for r in ref]))
        assert e.value.code == _lib.PS_EINVAL
        again = [r.copy() for r in ref]
        s.run(wl.views, again, p2, DepthSnapshot(8, 0, missing))
        _same(again, alt, "usable after PS_EINVAL")
    be.close()
