"""The allocation-free entry point (rtod_detect_window_static), for callers
that cannot allocate device memory while detecting (code inside a pool or
allocator it does not own, real-time loops that cannot afford cudaMalloc's
synchronisation, hosts that lend the library only their own buffers).

Called through the C ABI on device buffers the test owns; its output must
equal the outliers the regular entry point (rtod_run via Detector) reports for
the same windows, on two calls in a row (the shared scratch array keeps the
first call's contents, so the second call shows that it clears what it must).
Outlier IDs are integers, so "equal" is exact."""
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


def static_detect(torch, native, window_pts, R, K, pred=0):
    """One call of the allocation-free entry point on a device copy of the window."""
    dev = torch.from_numpy(np.ascontiguousarray(window_pts, np.float32)).cuda()
    n, dim = window_pts.shape
    out = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    n_out = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    rc = native.lib().rtod_detect_window_static(ctypes.c_void_p(dev.data_ptr()), n, dim, float(R), K, pred,
                                                ctypes.c_void_p(out.data_ptr()), ctypes.byref(n_out), None)
    native.check(rc)
    return out[:n_out.value].cpu().numpy()


@pytest.mark.parametrize("case", ["walk1d", "sensor3d"])
def test_static_entry_matches_regular_entry_on_two_calls(env, case):
    torch, rtod, native = env
    from rtod_b200 import datagen
    if case == "walk1d":
        pts = datagen.random_walk(60_000, 0.1, seed=21, jump_frac=0.005)
        W, S, R, K = 20_000, 2_000, 0.3, 20
    else:
        pts = datagen.sensor_3d(30_000, seed=22)
        W, S, R, K = 10_000, 500, 1.9, 50
    with rtod.Detector(W, S, R, K, dim=pts.shape[1]) as det:
        ref = det.run(pts, max_slides=6)
    for j in (0, 5):  # two calls in a row, on different windows
        lo = (j + 1) * S
        got = static_detect(torch, native, pts[lo:lo + W], R, K)
        np.testing.assert_array_equal(got, ref.slide(j) - lo)
    # and the first window again, after the scratch held another window
    got = static_detect(torch, native, pts[S:S + W], R, K)
    np.testing.assert_array_equal(got, ref.slide(0) - S)


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
