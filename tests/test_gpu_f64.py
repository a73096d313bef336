"""Double storage (rtod_config.coord = RTOD_COORD_F64): points passed, stored
and compared as doubles with RTOD's double predicate, the way RTOD keeps
double3 points (src/ods/optixScan.cpp:95-147) and tests them
(src/ods/optixScan.cu:170-190). Checked through the C ABI against the
double-storage golden fixtures and the oracle's double mode, on both
engines, push/detect and run; bit-exact."""
import os

import numpy as np
import pytest

from conftest import golden_cases_f64, load_golden

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


def det(rtod, W, S, R, K, dim, **kw):
    return rtod.Detector(W, S, R, K, dim=dim, pred="f64_lt", coord="f64", **kw)


@pytest.mark.parametrize("path", golden_cases_f64(), ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("engine,graph", [("window", True), ("window", False), ("span", True),
                                          ("window-group", True)])
def test_run_matches_double_golden(rtod, path, engine, graph):
    meta, pts, off, ids = load_golden(path)
    kw = dict(engine="window", count="group") if engine == "window-group" else dict(engine=engine)
    with det(rtod, meta["W"], meta["S"], meta["R"], meta["K"], pts.shape[1], use_graph=graph, **kw) as d:
        r = d.run(pts)
    np.testing.assert_array_equal(r.offsets, off)
    np.testing.assert_array_equal(r.ids, ids)


@pytest.mark.parametrize("path", golden_cases_f64(), ids=lambda p: os.path.basename(p)[:-4])
def test_push_detect_matches_double_golden(rtod, path):
    meta, pts, off, ids = load_golden(path)
    W, S = meta["W"], meta["S"]
    with det(rtod, W, S, meta["R"], meta["K"], pts.shape[1]) as d:
        d.push(pts[:W])
        for j in range(len(off) - 1):
            d.push(pts[W + j * S:W + (j + 1) * S])
            np.testing.assert_array_equal(d.detect(), ids[off[j]:off[j + 1]])


def jitter(x, seed):
    """Values that float32 cannot hold exactly."""
    return x.astype(np.float64) + np.random.default_rng(seed).uniform(-1e-9, 1e-9, x.shape)


@pytest.mark.parametrize("engine", ["span", "window"])
def test_stock_like_double_vs_oracle(rtod, oracle_mod, engine):
    from rtod_b200 import datagen
    w = datagen.stock_like()
    sl = 30
    pts = jitter(w.points[:w.window + sl * w.slide], 31)
    off, ids, _ = oracle_mod.detect(pts, w.window, w.slide, w.R, w.K, "f64_lt", threads=8, f64=True)
    with det(rtod, w.window, w.slide, w.R, w.K, 1, engine=engine) as d:
        r = d.run(pts)
    np.testing.assert_array_equal(r.offsets, off)
    np.testing.assert_array_equal(r.ids, ids)


@pytest.mark.parametrize("router", [False, True])
def test_sensor_like_double_vs_oracle(rtod, oracle_mod, router):
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    sl = 60
    pts = jitter(w.points[:w.window + sl * w.slide], 32)
    off, ids, _ = oracle_mod.detect(pts, w.window, w.slide, w.R, w.K, "f64_lt", threads=8, f64=True)
    with det(rtod, w.window, w.slide, w.R, w.K, 3, router=router) as d:
        r = d.run(pts)
    np.testing.assert_array_equal(r.offsets, off)
    np.testing.assert_array_equal(r.ids, ids)


def test_double_storage_of_float_values_equals_float_storage(rtod):
    """Whole stock-like stream: double storage of float32 values gives the
    double predicate's results on float storage (a size-independent check)."""
    from rtod_b200 import datagen
    w = datagen.stock_like()
    with rtod.Detector(w.window, w.slide, w.R, w.K, pred="f64_lt") as d:
        a = d.run(w.points)
    with det(rtod, w.window, w.slide, w.R, w.K, 1, batch=64) as d:
        b = d.run(w.points.astype(np.float64))
    np.testing.assert_array_equal(a.offsets, b.offsets)
    np.testing.assert_array_equal(a.ids, b.ids)


def test_device_double_tensor(rtod, oracle_mod):
    import torch
    meta, pts, off, ids = load_golden(golden_cases_f64()[-1])
    with det(rtod, meta["W"], meta["S"], meta["R"], meta["K"], pts.shape[1]) as d:
        r = d.run(torch.from_numpy(pts).cuda())
    np.testing.assert_array_equal(r.offsets, off)
    np.testing.assert_array_equal(r.ids, ids)


def test_coordinate_type_errors(rtod):
    import ctypes
    from rtod_b200 import _native
    with pytest.raises(rtod.RtodError):
        rtod.Detector(1000, 100, 0.5, 5, coord="f64")  # double storage needs the double predicate
    with det(rtod, 1000, 100, 0.5, 5, 1) as d:
        pts = np.zeros(1000, np.float32)
        rc = _native.lib().rtod_push_slide(d._h, pts.ctypes.data_as(ctypes.c_void_p), 1000)
        assert rc == -2 and b"double" in _native.lib().rtod_last_error()
    with rtod.Detector(1000, 100, 0.5, 5) as d:
        pts = np.zeros(1000, np.float64)
        rc = _native.lib().rtod_push_slide_f64(d._h, pts.ctypes.data_as(ctypes.c_void_p), 1000)
        assert rc == -2 and b"float" in _native.lib().rtod_last_error()


REF_CASES = sorted(__import__("glob").glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                                        "ref_*.npz")))


@pytest.mark.parametrize("path", REF_CASES, ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("engine", ["span", "window", "push"])
def test_matches_rtod_reference_run(rtod, path, engine):
    """Double storage against outliers produced by RTOD's own code
    (tests/golden/ref_*.npz: detect_outlier and check_outlier of
    src/ods/optixScan.cpp run on the same stream), every slide."""
    from test_reference_pin import load_ref
    meta, pts, off, ids = load_ref(path)
    pts = pts.astype(np.float64)
    W, S = meta["W"], meta["S"]
    with det(rtod, W, S, meta["R"], meta["K"], pts.shape[1],
             **({} if engine == "push" else dict(engine=engine))) as d:
        if engine == "push":
            d.push(pts[:W])
            for j in range(meta["slides"]):
                d.push(pts[W + j * S:W + (j + 1) * S])
                np.testing.assert_array_equal(d.detect(), ids[off[j]:off[j + 1]])
        else:
            r = d.run(pts)
            np.testing.assert_array_equal(r.offsets, off)
            np.testing.assert_array_equal(r.ids, ids)
