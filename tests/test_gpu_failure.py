"""Device-side failure detection without a fault: the scans' look-back wait
is run for a tile whose predecessor never publishes (a flag nothing sets).
The wait gives up after its bound, the kernel records the timeout and
returns, the host reads RTOD_ERR_TIMEOUT's device code, and the device keeps
working for the next detection."""
import ctypes

import numpy as np
import pytest

from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rtod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rtod_b200 import build
    build.build()
    import rtod_b200
    return rtod_b200


def test_bounded_wait_times_out_and_device_stays_usable(rtod):
    from rtod_b200 import _native
    L = _native.lib()
    for _ in range(2):
        t, ms = ctypes.c_int32(), ctypes.c_double()
        assert L.rtod_check_bounded_wait(0, ctypes.byref(t), ctypes.byref(ms)) == 0
        assert t.value == 1  # the wait ran out and said so
        assert 1.0 < ms.value < 20_000.0  # bounded: milliseconds to seconds, not forever
        meta, pts, off, ids = load_golden(golden_cases()[0])
        with rtod.Detector(meta["W"], meta["S"], meta["R"], meta["K"], dim=pts.shape[1],
                           pred=meta["pred"]) as det:
            r = det.run(pts)
        np.testing.assert_array_equal(r.offsets, off)
        np.testing.assert_array_equal(r.ids, ids)


def test_bounded_wait_bad_device(rtod):
    from rtod_b200 import _native
    L = _native.lib()
    t, ms = ctypes.c_int32(), ctypes.c_double()
    assert L.rtod_check_bounded_wait(999, ctypes.byref(t), ctypes.byref(ms)) == -8  # RTOD_ERR_NODEV
    assert t.value == 0
