"""The allocation-free median filter entry point, checked against the session's median filter.

`ps_median_filter_inplace_noalloc` serves callers that own device buffers but may not allocate device memory: a
host framework whose memory pool owns every allocation, a service that fixes its memory budget at start-up, or a
real-time loop where an allocation and its implicit synchronisation are not allowed.  Its input copy lives in a
static device array instead of a session buffer.  These tests call it through the C ABI, on device buffers the test
itself allocates (the test may allocate; the entry point must not), twice in a row on different planes, and require
the same bits as `ps_median_filter` (the tolerance of every parity test here is zero).

This file is named to be collected last, so a run that stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from cumulus3d_b200 import _lib, scenes
from cumulus3d_b200.patchstereo import KernelInput, KernelView, LevelImage, PatchMatchBackend, RunParams, ViewState

pytestmark = pytest.mark.gpu


def _noalloc(planes_dev, w: int, h: int, k, stream=None) -> int:
    kk = (C.c_float * 4)(*[float(x) for x in k])
    ptr = planes_dev.data_ptr() if isinstance(planes_dev, torch.Tensor) else planes_dev
    return _lib.engine().ps_median_filter_inplace_noalloc(0, C.c_void_p(ptr), w, h, kk,
                                                          None if stream is None else C.c_void_p(stream))


def _run_noalloc(state: ViewState, k, stream: "torch.cuda.Stream" = None) -> ViewState:
    planes = np.ascontiguousarray(state.planes(), np.float32)
    dev = torch.from_numpy(planes).cuda()
    torch.cuda.synchronize()
    if stream is None:
        assert _noalloc(dev, state.width, state.height, k) == _lib.PS_OK
        torch.cuda.synchronize()
    else:
        assert _noalloc(dev, state.width, state.height, k, stream.cuda_stream) == _lib.PS_OK
        stream.synchronize()
    out = dev.cpu().numpy()
    res = state.copy()
    res.normal[...] = out[..., :3]
    res.depth[...] = out[..., 3]
    return res


def test_noalloc_median_equals_session_median_twice():
    wl = scenes.workload_small(96, 64, views=3, window_radius=3, seed=41)
    be = PatchMatchBackend(0, math="parity")
    states = [ViewState.new(c.width, c.height) for c in wl.cams]
    with be.begin(wl.input) as s:
        s.run(wl.views, states, RunParams(0, False, True, 2, 1))
        want = s.median_filter(wl.input, 0, wl.views, states)
    be.close()
    for v in (0, 1, 0):  # consecutive calls on different planes share the static array
        got = _run_noalloc(states[v], wl.cams[v].k)
        np.testing.assert_array_equal(got.depth, want[v].depth)
        np.testing.assert_array_equal(got.normal, want[v].normal)
    # on a stream of the caller's own (ordered after that stream's earlier work), twice in a row
    side = torch.cuda.Stream()
    for v in (2, 1):
        got = _run_noalloc(states[v], wl.cams[v].k, side)
        np.testing.assert_array_equal(got.depth, want[v].depth)
        np.testing.assert_array_equal(got.normal, want[v].normal)


def test_noalloc_rejects_memory_it_cannot_filter():
    """Host memory (or memory of another device) is rejected before any device work, and the caller's current device
    is unchanged afterwards."""
    w, h = 16, 8
    k = (20.0, 20.0, 7.5, 3.5)
    host = np.zeros((h, w, 4), np.float32)
    dev_before = torch.cuda.current_device()
    assert _noalloc(host.ctypes.data, w, h, k) == _lib.PS_EINVAL
    assert torch.cuda.current_device() == dev_before
    dev = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    assert _noalloc(dev, w, h, k) == _lib.PS_OK
    torch.cuda.synchronize()
    assert torch.cuda.current_device() == dev_before


def test_noalloc_tall_image():
    """A two-column image taller than a session accepts (sessions take sides up to 32768) and taller than 65535
    blocks of 8 rows: the entry point's one-dimensional launch covers it.  The reference is the CPU restatement of the
    median filter, which the parity tests hold equal to the session's."""
    from oracle import oracle
    w, h = 2, 1 << 20
    k = (500.0, 500.0, 0.5, h / 2.0)
    s = ViewState.new(w, h)
    rng = np.random.default_rng(3)
    n = rng.normal(0.0, 0.1, (h, w, 3)).astype(np.float32) + np.float32([0.0, 0.0, -1.0])
    s.normal[...] = n / np.linalg.norm(n, axis=-1, keepdims=True)
    s.depth[...] = rng.uniform(25.0, 60.0, (h, w)).astype(np.float32)
    inp = KernelInput([KernelView(1, [LevelImage(np.zeros((h, w), np.float32), k)], [], [], 20.0, 80.0)], 1)
    want = oracle.median(inp, 0, [0], [s])[0]
    got = _run_noalloc(s, k)
    np.testing.assert_array_equal(got.depth, want.depth)
    np.testing.assert_array_equal(got.normal, want.normal)


def test_noalloc_median_full_hd_and_size_limit():
    w, h = 1920, 1080
    assert w * h <= _lib.PS_NOALLOC_MAX_PIXELS  # a full-HD image fits the static array
    f = (w / 2.0) / np.tan(np.radians(30.0))
    k = (f, f, (w - 1) / 2.0, (h - 1) / 2.0)
    inp = KernelInput([KernelView(1, [LevelImage(np.zeros((h, w), np.float32), k)], [], [], 20.0, 80.0)], 1)
    rng = np.random.default_rng(7)
    st = []
    for _ in range(2):
        s = ViewState.new(w, h)
        n = rng.normal(0.0, 0.15, (h, w, 3)).astype(np.float32) + np.float32([0.0, 0.0, -1.0])
        s.normal[...] = n / np.linalg.norm(n, axis=-1, keepdims=True)
        s.depth[...] = rng.uniform(25.0, 60.0, (h, w)).astype(np.float32)
        s.depth[rng.random((h, w)) < 0.1] = 0.0  # some invalid pixels pass through
        st.append(s)
    be = PatchMatchBackend(0, math="parity")
    with be.begin(inp) as sess:
        want = [sess.median_filter(inp, 0, [0], [s])[0] for s in st]
    be.close()
    for s, ref in zip(st, want):
        got = _run_noalloc(s, k)
        np.testing.assert_array_equal(got.depth, ref.depth)
        np.testing.assert_array_equal(got.normal, ref.normal)
    # beyond the static array's capacity: rejected before any device work
    dev = torch.zeros(16, dtype=torch.float32, device="cuda")
    too_wide = (_lib.PS_NOALLOC_MAX_PIXELS // 1024) + 1
    assert _noalloc(dev, too_wide, 1024, k) == _lib.PS_EINVAL
