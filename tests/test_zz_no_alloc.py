"""The allocation-free entry point (rtod_detect_window_static), for callers
that cannot allocate device memory while detecting (code inside a pool or
allocator it does not own, real-time loops that cannot afford cudaMalloc's
synchronisation, hosts that lend the library only their own buffers).

Called through the C ABI on device buffers the test owns. Its outliers must
equal those of the regular entry point (rtod_run via Detector) and of the CPU
oracle for the same windows, on calls in a row (the shared scratch array
keeps each call's contents, so later calls show that it clears what it
must), under both predicates, for K = 0 and K >= n, and after a call that
failed part-way on bad input. Outlier IDs are integers, so "equal" is exact.
This file is collected last so that a run stopping at the first failure has
run every other test before it."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rtod_b200 import build
    build.build()
    import rtod_b200
    from rtod_b200 import _native
    return torch, rtod_b200, _native


class Static:
    """Device buffers owned by the caller, reused for every call."""

    def __init__(self, torch, native, n_max=65536, dim_max=3):
        self.torch, self.native = torch, native
        self.pts = torch.zeros((n_max * dim_max,), dtype=torch.float32, device="cuda")
        self.out = torch.zeros((n_max,), dtype=torch.int64, device="cuda")

    def call(self, window_pts, R, K, pred=0):
        """Returns (return code, outlier offsets or None)."""
        w = np.ascontiguousarray(window_pts, np.float32)
        n, dim = w.shape
        self.pts[:n * dim].copy_(self.torch.from_numpy(w.ravel()))
        self.out.fill_(-1)
        n_out = ctypes.c_int64(-1)
        self.torch.cuda.synchronize()
        rc = self.native.lib().rtod_detect_window_static(
            ctypes.c_void_p(self.pts.data_ptr()), n, dim, float(R), K, pred,
            ctypes.c_void_p(self.out.data_ptr()), ctypes.byref(n_out), None)
        if rc != 0:
            return rc, None
        return rc, self.out[:n_out.value].cpu().numpy()


def oracle_window(oracle_mod, pts, R, K, pred="fp32_le"):
    """The oracle's outliers of one window holding all of pts (W = S = n)."""
    n = pts.shape[0]
    both = np.concatenate([pts, pts])  # one slide: the window [n, 2n) equals pts
    off, ids, _ = oracle_mod.detect(both, n, n, R, K, pred, engine="grid", threads=8)
    return ids[off[0]:off[1]] - n


@pytest.mark.parametrize("case", ["walk1d", "sensor3d"])
def test_static_entry_matches_regular_entry_on_two_calls(env, oracle_mod, case):
    torch, rtod, native = env
    from rtod_b200 import datagen
    if case == "walk1d":
        pts = datagen.random_walk(60_000, 0.1, seed=21, jump_frac=0.005)
        W, S, R, K = 20_000, 2_000, 0.3, 20
    else:
        pts = datagen.sensor_3d(30_000, seed=22)
        W, S, R, K = 10_000, 500, 1.9, 50
    st = Static(torch, native)
    with rtod.Detector(W, S, R, K, dim=pts.shape[1]) as det:
        ref = det.run(pts, max_slides=6)
    for j in (0, 5):  # two calls in a row, on different windows
        lo = (j + 1) * S
        rc, got = st.call(pts[lo:lo + W], R, K)
        assert rc == 0
        np.testing.assert_array_equal(got, ref.slide(j) - lo)
        np.testing.assert_array_equal(got, oracle_window(oracle_mod, pts[lo:lo + W], R, K))
    # and the first window again, after the scratch held another window
    rc, got = st.call(pts[S:S + W], R, K)
    np.testing.assert_array_equal(got, ref.slide(0) - S)


@pytest.mark.parametrize("dim", [1, 3])
def test_static_entry_predicates_and_K_edges(env, oracle_mod, dim):
    """Both predicates, K = 0 (only isolated points are outliers) and K >= n
    (every point is an outlier), each against the oracle, calls in a row."""
    torch, rtod, native = env
    from rtod_b200 import datagen
    st = Static(torch, native)
    if dim == 1:
        pts = datagen.random_walk(8_000, 0.1, seed=31, jump_frac=0.01)
        R = 0.05
    else:
        pts = datagen.sensor_3d(8_000, seed=32)
        R = 0.9
    for pred_name, pred in (("fp32_le", 0), ("f64_lt", 1)):
        for K in (0, 7, 8_000, 9_000):
            rc, got = st.call(pts, R, K, pred)
            assert rc == 0
            expect = oracle_window(oracle_mod, pts, R, K, pred_name)
            np.testing.assert_array_equal(got, expect, err_msg=f"{pred_name} K={K}")
            if K >= len(pts):
                assert len(got) == len(pts)


def test_static_entry_after_a_failed_call(env, oracle_mod):
    """A call that stops on bad input (a NaN, a coordinate too large for the
    grid) leaves the shared array part-way through a detection; the next
    valid call must still match the oracle exactly."""
    torch, rtod, native = env
    from rtod_b200 import datagen
    st = Static(torch, native)
    pts = datagen.random_walk(20_000, 0.1, seed=41, jump_frac=0.005)
    R, K = 0.3, 20
    bad = pts.copy()
    bad[7_777, 0] = np.nan
    rc, _ = st.call(bad, R, K)
    assert rc == -5  # RTOD_ERR_INPUT
    rc, got = st.call(pts, R, K)
    assert rc == 0
    np.testing.assert_array_equal(got, oracle_window(oracle_mod, pts, R, K))
    huge = pts.copy()
    huge[123, 0] = 3e30
    rc, _ = st.call(huge, 1e-6, K)
    assert rc == -5
    rc, got = st.call(pts[:12_000], R, K)
    assert rc == 0
    np.testing.assert_array_equal(got, oracle_window(oracle_mod, pts[:12_000], R, K))


def test_static_entry_allocates_nothing(env):
    """After a first call (which also loads the kernels), repeated calls leave
    the device's free memory unchanged."""
    torch, rtod, native = env
    from rtod_b200 import datagen
    st = Static(torch, native)
    pts = datagen.random_walk(65_536, 0.1, seed=51, jump_frac=0.005)
    assert st.call(pts, 0.3, 20)[0] == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for K in (5, 20, 50):
        assert st.call(pts, 0.3, K)[0] == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_entry_rejects_sizes_beyond_its_maximum(env):
    torch, rtod, native = env
    L = native.lib()
    big = torch.zeros((65537, 1), dtype=torch.float32, device="cuda")
    out = torch.zeros(65537, dtype=torch.int64, device="cuda")
    n_out = ctypes.c_int64(0)
    rc = L.rtod_detect_window_static(ctypes.c_void_p(big.data_ptr()), 65537, 1, 1.0, 5, 0,
                                     ctypes.c_void_p(out.data_ptr()), ctypes.byref(n_out), None)
    assert rc == -4 and b"1..65536" in L.rtod_last_error()
    rc = L.rtod_detect_window_static(ctypes.c_void_p(big.data_ptr()), 100, 4, 1.0, 5, 0,
                                     ctypes.c_void_p(out.data_ptr()), ctypes.byref(n_out), None)
    assert rc == -4
