"""Group counts (rtod_config.count = RTOD_COUNT_GROUP, and the span engine's
count): one warp per cell bin, its points sharing the stencil's candidates,
with idle lanes refilled from the group and every point walking the
candidate chunks once around from where it joined. Checked bit-exact
against the golden fixtures and the CPU oracle, including groups far larger
than a warp (8-d Gaussian blobs: no cell is ever all-inlier and the
projected stencil holds most of a blob), stencils of several 32-slot rounds
(3-d with 2 and 3 cells per R) and the multi-stream API."""
import os

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


def assert_same(res, off, ids):
    np.testing.assert_array_equal(res.offsets, off)
    np.testing.assert_array_equal(res.ids, ids)


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("opt,graph,n", [(2, True, 0), (0, False, 0), (1, True, 3)])
def test_run_group_matches_golden(rtod, path, opt, graph, n):
    meta, pts, off, ids = load_golden(path)
    with rtod.Detector(meta["W"], meta["S"], meta["R"], meta["K"], dim=pts.shape[1], opt=opt,
                       pred=meta["pred"], use_graph=graph, cells_per_r=n, engine="window",
                       count="group") as det:
        assert_same(det.run(pts), off, ids)
        assert det.count_mode == "group"


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_push_detect_group_matches_golden(rtod, path):
    meta, pts, off, ids = load_golden(path)
    W, S = meta["W"], meta["S"]
    with rtod.Detector(W, S, meta["R"], meta["K"], dim=pts.shape[1], pred=meta["pred"], count="group") as det:
        det.push(pts[:W])
        for j in range(len(off) - 1):
            det.push(pts[W + j * S:W + (j + 1) * S])
            np.testing.assert_array_equal(det.detect(), ids[off[j]:off[j + 1]])


def oracle_run(oracle_mod, pts, W, S, R, K, slides, pred="fp32_le"):
    pts = pts[:W + slides * S]
    off, ids, _ = oracle_mod.detect(pts, W, S, R, K, pred, engine="grid", threads=8)
    return pts, off, ids


@pytest.mark.parametrize("kw", [dict(engine="window", count="group"), dict(engine="window", count="point"),
                                dict(engine="span"), dict(engine="window"),
                                dict(engine="window", router=True)])
def test_8d_gaussian_blobs(rtod, oracle_mod, kw):
    """8-d mixture: cells hold hundreds of points, all counted."""
    from rtod_b200 import datagen
    W, S, K = 6000, 600, 20
    pts = datagen.gaussian_mixture(W + 6 * S, seed=61, dim=8)
    pts, off, ids = oracle_run(oracle_mod, pts, W, S, 0.05, K, 6)
    assert len(ids) > 6 * 30  # tail points and noise
    with rtod.Detector(W, S, 0.05, K, dim=8, **kw) as det:
        assert_same(det.run(pts), off, ids)
        if kw.get("engine") == "window":
            # auto: point counts for a window this small
            assert det.count_mode == kw.get("count", "point")


def test_auto_count_mode(rtod):
    # group counts in more than 3 dimensions once a window holds >= 4096 points per SM
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    W = -(-4096 * sms // 20) * 20  # a multiple of the slide W/20
    for d, router, want in ((8, False, "group"), (8, True, "point"), (3, False, "point")):
        with rtod.Detector(W, W // 20, 0.1, 50, dim=d, router=router) as det:
            assert det.count_mode == want
    W2 = (W // 2) // 20 * 20
    with rtod.Detector(W2, W2 // 20, 0.1, 50, dim=8) as det:
        assert det.count_mode == "point"


@pytest.mark.parametrize("n", [1, 2, 3])
@pytest.mark.parametrize("engine", ["window", "span"])
def test_3d_stencil_rounds(rtod, oracle_mod, n, engine):
    """27, 125 and 343 stencil slots: one to eleven rounds of 32 slots."""
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    pts, off, ids = oracle_run(oracle_mod, w.points, w.window, w.slide, w.R, w.K, 25)
    kw = dict(count="group") if engine == "window" else {}
    with rtod.Detector(w.window, w.slide, w.R, w.K, dim=3, cells_per_r=n, engine=engine, **kw) as det:
        assert_same(det.run(pts), off, ids)


def test_1d_group_counts(rtod, oracle_mod):
    from rtod_b200 import datagen
    w = datagen.stock_like()
    pts, off, ids = oracle_run(oracle_mod, w.points, w.window, w.slide, w.R, w.K, 10)
    for n in (1, 2, 4):
        with rtod.Detector(w.window, w.slide, w.R, w.K, cells_per_r=n, engine="window", count="group") as det:
            assert_same(det.run(pts), off, ids)


@pytest.mark.parametrize("K", [0, 1, 5000])
def test_group_extremes(rtod, oracle_mod, K):
    """K = 0 (no outliers: a point counts itself), K = 1, and K at least the
    window (every point an outlier without a test)."""
    from rtod_b200 import datagen
    W, S = 5000, 500
    pts = datagen.gaussian_mixture(W + 4 * S, seed=62, dim=5)
    pts, off, ids = oracle_run(oracle_mod, pts, W, S, 0.06, K, 4)
    with rtod.Detector(W, S, 0.06, K, dim=5, count="group", engine="window") as det:
        assert_same(det.run(pts), off, ids)


def test_double_predicate_group(rtod, oracle_mod):
    from rtod_b200 import datagen
    W, S = 4000, 400
    pts = datagen.random_walk(W + 5 * S, 0.1, seed=63, dim=4)
    pts, off, ids = oracle_run(oracle_mod, pts, W, S, 0.35, 15, 5, pred="f64_lt")
    with rtod.Detector(W, S, 0.35, 15, dim=4, pred="f64_lt", count="group", engine="window") as det:
        assert_same(det.run(pts), off, ids)


def test_router_is_bypassed_in_group_mode(rtod, oracle_mod):
    from rtod_b200 import datagen
    W, S = 5000, 500
    pts = datagen.random_walk(W + 5 * S, 0.1, seed=64, dim=3)
    pts, off, ids = oracle_run(oracle_mod, pts, W, S, 0.3, 20, 5)
    with rtod.Detector(W, S, 0.3, 20, dim=3, router=True, count="group") as det:
        assert_same(det.run(pts), off, ids)
        info = det.router_info()
        assert info["routed_early"] == 0 and info["routed_sweep"] == 0


def test_count_mode_config_errors(rtod):
    with pytest.raises(KeyError):
        rtod.Detector(1000, 100, 0.5, 5, count="fast")
    import ctypes
    from rtod_b200 import _native
    cfg = _native.Config()
    _native.lib().rtod_config_init(ctypes.byref(cfg))
    cfg.count = 7
    h = ctypes.c_void_p()
    assert _native.lib().rtod_create(ctypes.byref(cfg), ctypes.byref(h)) != 0
    assert b"count" in _native.lib().rtod_last_error()
