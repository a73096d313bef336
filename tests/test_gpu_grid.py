"""GPU parity of the streaming grid engine of push/detect (the cell grid of
the window kept on the device, each bin a FIFO that a slide's expiry and
insertion update in place): slide by slide against the golden fixtures and
the CPU oracle, bit-exact, through its growth, rebuild and fallback paths."""
import os

import numpy as np
import pytest

from conftest import golden_cases, golden_cases_f64, load_golden

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


def stream(det, pts, W, S, slides):
    """RTOD's per-slide loop through the detector: the IDs of every slide."""
    det.push(pts[:W])
    out = []
    for j in range(slides):
        det.push(pts[W + j * S:W + (j + 1) * S])
        out.append(det.detect())
    return out


def expect(oracle_mod, pts, W, S, R, K, slides, pred="fp32_le", f64=False):
    off, ids, _ = oracle_mod.detect(pts[:W + slides * S], W, S, R, K, pred, engine="grid",
                                    threads=os.cpu_count() or 4, f64=f64)
    return [ids[off[j]:off[j + 1]] for j in range(slides)]


def assert_slides(got, want):
    assert len(got) == len(want)
    for j, (g, w) in enumerate(zip(got, want)):
        np.testing.assert_array_equal(g, w, err_msg=f"slide {j}")


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("kw", [dict(), dict(opt=0), dict(cells_per_r=1), dict(cells_per_r=3),
                                dict(use_graph=False)], ids=["default", "opt0", "n1", "n3", "nograph"])
def test_grid_matches_golden(rtod, path, kw):
    meta, pts, off, ids = load_golden(path)
    W, S = meta["W"], meta["S"]
    if kw.get("cells_per_r") == 3 and pts.shape[1] > 3:
        pytest.skip("cells_per_r is at most 3 beyond 1-d")
    with rtod.Detector(W, S, meta["R"], meta["K"], dim=pts.shape[1], pred=meta["pred"], engine="grid",
                       **kw) as det:
        got = stream(det, pts, W, S, len(off) - 1)
        assert det.stream_engine["engine"] == ("grid" if pts.shape[1] <= 3 else "window")
    assert_slides(got, [ids[off[j]:off[j + 1]] for j in range(len(off) - 1)])


@pytest.mark.parametrize("path", golden_cases_f64(), ids=lambda p: os.path.basename(p)[:-4])
def test_grid_double_storage_matches_golden(rtod, path):
    meta, pts, off, ids = load_golden(path)
    W, S = meta["W"], meta["S"]
    with rtod.Detector(W, S, meta["R"], meta["K"], dim=pts.shape[1], pred="f64_lt", coord="f64",
                       engine="grid") as det:
        got = stream(det, pts, W, S, len(off) - 1)
        assert det.stream_engine["engine"] == "grid"
    assert_slides(got, [ids[off[j]:off[j + 1]] for j in range(len(off) - 1)])


def test_grid_runs_where_requested_and_applicable(rtod):
    cases = [(dict(), 1, "window"), (dict(), 3, "window"), (dict(engine="grid"), 1, "grid"),
             (dict(engine="grid"), 3, "grid"), (dict(engine="grid"), 8, "window"),
             (dict(engine="window"), 1, "window"), (dict(engine="span"), 1, "window"),
             (dict(engine="grid", router=True), 1, "grid")]
    for kw, dim, want in cases:
        with rtod.Detector(2000, 100, 0.5, 10, dim=dim, **kw) as det:
            assert det.stream_engine["engine"] == want, (kw, dim)


def test_grid_stock_like_full_stream(rtod, oracle_mod):
    """Every slide of the stock-like stream (W=100k, S=5k, 189 slides) through
    push/detect; the random walk keeps entering new cells (bins grow)."""
    from rtod_b200 import datagen
    w = datagen.stock_like()
    want = expect(oracle_mod, w.points, w.window, w.slide, w.R, w.K, w.slides)
    with rtod.Detector(w.window, w.slide, w.R, w.K, engine="grid") as det:
        got = stream(det, w.points, w.window, w.slide, w.slides)
        info = det.stream_engine
        assert info["engine"] == "grid" and info["builds"] == 1 and info["max_occ"] > 0
    assert_slides(got, want)


@pytest.mark.parametrize("pred", ["fp32_le", "f64_lt"])
def test_grid_sensor_like(rtod, oracle_mod, pred):
    """3-d sensor-like stream (uniform outliers in [-30, 30]^3: the window's
    cells alias in the 3-d bin map), 300 slides."""
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    want = expect(oracle_mod, w.points, w.window, w.slide, w.R, w.K, 300, pred)
    with rtod.Detector(w.window, w.slide, w.R, w.K, dim=3, pred=pred, engine="grid") as det:
        got = stream(det, w.points, w.window, w.slide, 300)
        assert det.stream_engine["engine"] == "grid"
    assert_slides(got, want)


@pytest.mark.parametrize("K", [30, 70])
def test_grid_dense_bins(rtod, oracle_mod, K):
    """Gaussian mixture (W=100k, R=0.028): bins of thousands of points beside
    sparse ones; 40 slides."""
    from rtod_b200 import datagen
    w = datagen.gaussian_like(K)
    want = expect(oracle_mod, w.points, w.window, w.slide, w.R, w.K, 40)
    with rtod.Detector(w.window, w.slide, w.R, w.K, engine="grid") as det:
        got = stream(det, w.points, w.window, w.slide, 40)
        assert det.stream_engine["max_occ"] > 1000
    assert_slides(got, want)


@pytest.mark.parametrize("pool", [1024, 8192])
def test_grid_rebuilds_when_its_pool_runs_out(rtod, oracle_mod, pool):
    """A pool far too small for the stream: the first build doubles it until
    the regions fit, later growth exhausts it, and each detection that runs
    out rebuilds the grid from the ring and counts again."""
    from rtod_b200 import datagen
    pts = datagen.random_walk(40_000, 0.3, seed=11, jump_frac=0.01)
    W, S, R, K, slides = 4000, 200, 0.4, 12, 180
    want = expect(oracle_mod, pts, W, S, R, K, slides)
    with rtod.Detector(W, S, R, K, cells_per_r=3, engine="grid") as det:
        det.set_grid_pool(pool)
        got = stream(det, pts, W, S, slides)
        info = det.stream_engine
        assert info["engine"] == "grid"
        assert info["builds"] > 1
    assert_slides(got, want)


def test_grid_aliased_bins_1d(rtod, oracle_mod):
    """A 1-d window spanning far more than the 65536 bins (cells of 1e-3 over
    a range of 1000): different cells share bins, the all-inlier rule is
    decided per bin."""
    rng = np.random.Generator(np.random.PCG64(5))
    base = rng.uniform(0.0, 1000.0, size=300).astype(np.float32)
    pts = (base[rng.integers(0, 300, size=30_000)] + rng.normal(0, 2e-3, size=30_000)).astype(np.float32)
    W, S, R, K, slides = 6000, 300, 2e-3, 8, 60
    want = expect(oracle_mod, pts, W, S, R, K, slides)
    with rtod.Detector(W, S, R, K, engine="grid") as det:
        got = stream(det, pts, W, S, slides)
    assert_slides(got, want)


def test_grid_matches_window_engine_and_run(rtod):
    """The same stream through the grid engine, the window engine and
    rtod_run: identical per-slide outliers."""
    from rtod_b200 import datagen
    pts = datagen.random_walk(60_000, 0.1, seed=12, jump_frac=0.005, dim=2)
    W, S, R, K = 10_000, 500, 0.3, 25
    slides = (len(pts) - W) // S
    with rtod.Detector(W, S, R, K, dim=2, engine="grid") as det:
        grid = stream(det, pts, W, S, slides)
    with rtod.Detector(W, S, R, K, dim=2, engine="window") as det:
        win = stream(det, pts, W, S, slides)
    with rtod.Detector(W, S, R, K, dim=2) as det:
        r = det.run(pts)
    assert_slides(grid, win)
    assert_slides(grid, [r.ids[r.offsets[j]:r.offsets[j + 1]] for j in range(slides)])


@pytest.mark.parametrize("K", [0, 5000])
def test_grid_k_edges(rtod, oracle_mod, K):
    from rtod_b200 import datagen
    pts = datagen.random_walk(12_000, 0.1, seed=13, jump_frac=0.01)
    W, S, R, slides = 4000, 400, 0.2, 20
    want = expect(oracle_mod, pts, W, S, R, K, slides)
    with rtod.Detector(W, S, R, K, engine="grid") as det:
        got = stream(det, pts, W, S, slides)
    assert_slides(got, want)


def test_grid_input_error_then_reset(rtod, oracle_mod):
    """A non-finite coordinate in a slide: RTOD_ERR_INPUT and the handle is
    poisoned; after rtod_reset the same handle streams correctly again."""
    from rtod_b200 import RtodError, datagen
    pts = datagen.random_walk(8_000, 0.1, seed=14, jump_frac=0.01)
    W, S, R, K, slides = 2000, 200, 0.3, 10, 30
    want = expect(oracle_mod, pts, W, S, R, K, slides)
    with rtod.Detector(W, S, R, K, engine="grid") as det:
        det.push(pts[:W])
        bad = pts[W:W + S].copy()
        bad[7] = np.nan
        det.push(bad)
        with pytest.raises(RtodError):
            det.detect()
        det.reset()
        got = stream(det, pts, W, S, slides)
        assert det.stream_engine["engine"] == "grid"
    assert_slides(got, want)
