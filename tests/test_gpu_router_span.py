"""The learned router in the span engine: runs of a bin's windows routed
either to independent early-exit counts or to delta segments (a window's
counts from the previous window's count bounds and the two changed slide
blocks). The exact count always decides, so every routing gives the
oracle's outliers bit for bit; these tests force each path, and let the
trained network route, on whole streams."""
import os

import numpy as np
import pytest

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


def expect(oracle_mod, w, pred="fp32_le", slides=None, f64=False):
    n = w.slides if slides is None else slides
    pts = w.points[:w.window + n * w.slide]
    if f64:
        pts = pts.astype(np.float64)
    return oracle_mod.detect(pts, w.window, w.slide, w.R, w.K, pred, engine="grid",
                             threads=os.cpu_count() or 4, f64=f64)[:2]


def workloads():
    from rtod_b200 import datagen
    return {"stock": datagen.stock_like(), "gau30": datagen.gaussian_like(30), "gau70": datagen.gaussian_like(70),
            "sensor": datagen.sensor_like(), "walk": datagen.small_walk()}


@pytest.mark.parametrize("name", ["stock", "gau30", "gau70", "sensor", "walk"])
@pytest.mark.parametrize("threshold", [2.0, 0.0, 0.5])
def test_routing_is_exact_on_whole_streams(rtod, oracle_mod, name, threshold):
    """threshold 2.0: every eligible run goes to a delta segment; 0.0: every
    count is independent; 0.5: the network routes (trained on the passes
    before). Three passes each, all slides."""
    w = workloads()[name]
    off, ids = expect(oracle_mod, w)
    with rtod.Detector(w.window, w.slide, w.R, w.K, dim=w.dim, engine="span", router=True,
                       cells_per_r=(3 if w.dim == 1 else 1)) as det:
        det.set_router_threshold(threshold)
        for _ in range(3):
            det.reset()
            r = det.run(w.points)
            np.testing.assert_array_equal(r.offsets, off)
            np.testing.assert_array_equal(r.ids, ids)
        info = det.router_info()
        if threshold == 2.0:
            assert info["routed_sweep"] > 0
        if threshold == 0.0:
            assert info["routed_sweep"] == 0


@pytest.mark.parametrize("kw", [dict(cells_per_r=2), dict(cells_per_r=6), dict(cells_per_r=8), dict(batch=7),
                                dict(batch=1), dict(use_graph=False), dict(pred="f64_lt"),
                                dict(block_warps=2)])
def test_delta_segments_across_settings(rtod, oracle_mod, kw):
    """Delta segments everywhere on the Gaussian-mixture stream (K = 30: most
    counted points are outliers) under other grids, batch sizes (segments
    cut at batch ends), launch modes and the double predicate."""
    from rtod_b200 import datagen
    w = datagen.gaussian_like(30)
    kw = dict(kw)
    pred = kw.pop("pred", "fp32_le")
    off, ids = expect(oracle_mod, w, pred, slides=60)
    with rtod.Detector(w.window, w.slide, w.R, w.K, engine="span", router=True, pred=pred, **kw) as det:
        det.set_router_threshold(2.0)
        r = det.run(w.points[:w.window + 60 * w.slide])
        np.testing.assert_array_equal(r.offsets, off)
        np.testing.assert_array_equal(r.ids, ids)


def test_delta_segments_double_storage(rtod):
    """Double storage with RTOD's double test against RTOD's own outliers
    (reference-run fixtures), delta segments everywhere."""
    from test_reference_pin import REF_CASES, load_ref
    for path in REF_CASES:
        meta, pts, off, ids = load_ref(path)
        with rtod.Detector(meta["W"], meta["S"], meta["R"], meta["K"], dim=pts.shape[1], pred="f64_lt",
                           coord="f64", engine="span", router=True) as det:
            det.set_router_threshold(2.0)
            r = det.run(pts.astype(np.float64))
            np.testing.assert_array_equal(r.offsets, off, err_msg=path)
            np.testing.assert_array_equal(r.ids, ids, err_msg=path)


def test_router_trains_on_span_counts(rtod, oracle_mod):
    """The span engine's counts train the network: after some passes it has
    taken Adam steps with a finite loss, and on the 3-d sensor-like stream
    (every point counted against large stencils, where delta segments cost
    less) it routes runs to delta segments; results stay exact throughout."""
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    off, ids = expect(oracle_mod, w, slides=300)
    pts = w.points[:w.window + 300 * w.slide]
    with rtod.Detector(w.window, w.slide, w.R, w.K, dim=3, engine="span", router=True, cells_per_r=1) as det:
        for _ in range(30):
            det.reset()
            r = det.run(pts)
            np.testing.assert_array_equal(r.offsets, off)
            np.testing.assert_array_equal(r.ids, ids)
        info = det.router_info()
        assert info["steps"] > 0 and np.isfinite(info["last_loss"])
        before = info["routed_sweep"]
        det.reset()
        det.run(pts)
        assert det.router_info()["routed_sweep"] > before
