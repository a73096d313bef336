"""The span engine (one counting sort per batch of windows) against the CPU
oracle and against the window engine, on the cases where its layout differs
from one sort per window: spans whose cells share bins, many slide blocks per
window, batches of one window, every point an outlier, the grid filter off,
the double predicate, 2-d/3-d/8-d stencils (one or several rounds of 32
cells), and the fall-back to the window engine when a window holds more
slide blocks than a span table allows. Bit-exact."""
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


def run(rtod, pts, W, S, R, K, slides, **kw):
    pts = pts[:W + slides * S]
    dim = pts.shape[1] if pts.ndim == 2 else 1
    with rtod.Detector(W, S, R, K, dim=dim, **kw) as det:
        res = det.run(pts)
        return res, det.tuning


def check_vs_oracle(rtod, oracle_mod, pts, W, S, R, K, slides, pred="fp32_le", **kw):
    off, ids, _ = oracle_mod.detect(pts[:W + slides * S], W, S, R, K, pred, engine="grid", threads=8)
    res, tun = run(rtod, pts, W, S, R, K, slides, pred=pred, engine="span", **kw)
    assert tun["engine"] == "span"
    np.testing.assert_array_equal(res.offsets, off)
    np.testing.assert_array_equal(res.ids, ids)
    return res


def test_cells_sharing_bins(rtod, oracle_mod):
    """Span key range far above 65536 cells, so that bins hold several cells:
    tight clusters (dense cells) among uniform points over a wide range."""
    rng = np.random.default_rng(71)
    n = 40_000
    centres = rng.uniform(0, 5000, 60)
    clustered = centres[rng.integers(0, 60, n)] + rng.normal(0, 5e-4, n)
    uniform = rng.uniform(0, 5000, n)
    pts = np.where(rng.random(n) < 0.6, clustered, uniform).astype(np.float32)[:, None]
    R = 0.004  # cells of R/2 = 0.002: about 2.5 million cells over the range
    for nc in (2, 5):
        check_vs_oracle(rtod, oracle_mod, pts, 8000, 400, R, 20, 40, cells_per_r=nc, batch=16)


def test_many_blocks_per_window(rtod, oracle_mod):
    from rtod_b200 import datagen
    pts = datagen.random_walk(30_000, 0.1, seed=72, jump_frac=0.005)
    check_vs_oracle(rtod, oracle_mod, pts, 6000, 30, 0.3, 15, 300, batch=64)


def test_batch_of_one_and_ragged_last_batch(rtod, oracle_mod):
    from rtod_b200 import datagen
    pts = datagen.random_walk(30_000, 0.1, seed=73, jump_frac=0.005)
    check_vs_oracle(rtod, oracle_mod, pts, 5000, 500, 0.3, 12, 45, batch=1)
    check_vs_oracle(rtod, oracle_mod, pts, 5000, 500, 0.3, 12, 45, batch=7)


def test_all_outliers_and_filter_off(rtod, oracle_mod):
    from rtod_b200 import datagen
    pts = datagen.random_walk(20_000, 0.1, seed=74)
    res = check_vs_oracle(rtod, oracle_mod, pts, 4000, 400, 0.3, 4000, 20)
    assert res.offsets[-1] == 20 * 4000  # K >= W: every window point is an outlier
    check_vs_oracle(rtod, oracle_mod, pts, 4000, 400, 0.3, 10, 20, opt=0)


def test_double_predicate(rtod, oracle_mod):
    from rtod_b200 import datagen
    w = datagen.stock_like()
    check_vs_oracle(rtod, oracle_mod, w.points, w.window, w.slide, w.R, w.K, 40, pred="f64_lt")


def test_full_stream_span_equals_window(rtod):
    """Whole stock-like stream: span and window engines, several grids."""
    from rtod_b200 import datagen
    w = datagen.stock_like()
    base, _ = run(rtod, w.points, w.window, w.slide, w.R, w.K, w.slides, engine="window")
    for kw in (dict(), dict(cells_per_r=1), dict(cells_per_r=3), dict(cells_per_r=6, batch=64),
               dict(use_graph=False, batch=9)):
        got, tun = run(rtod, w.points, w.window, w.slide, w.R, w.K, w.slides, engine="span", **kw)
        assert tun["engine"] == "span"
        np.testing.assert_array_equal(got.offsets, base.offsets)
        np.testing.assert_array_equal(got.ids, base.ids)


def test_too_many_blocks_falls_back_to_window_engine(rtod, oracle_mod):
    from rtod_b200 import datagen
    pts = datagen.random_walk(24_000, 0.1, seed=75, jump_frac=0.005)
    W, S = 20_480, 10  # 2048 slide blocks per window
    off, ids, _ = oracle_mod.detect(pts[:W + 5 * S], W, S, 0.3, 20, engine="grid", threads=8)
    res, tun = run(rtod, pts, W, S, 0.3, 20, 5, engine="span")
    assert tun["engine"] == "window"
    np.testing.assert_array_equal(res.offsets, off)
    np.testing.assert_array_equal(res.ids, ids)


def test_engine_auto_with_tuner(rtod):
    from rtod_b200 import datagen
    w = datagen.stock_like()
    base, _ = run(rtod, w.points, w.window, w.slide, w.R, w.K, 60, engine="window")
    got, tun = run(rtod, w.points, w.window, w.slide, w.R, w.K, 60, tuner=True)
    assert tun["engine"] in ("span", "window")
    np.testing.assert_array_equal(got.offsets, base.offsets)
    np.testing.assert_array_equal(got.ids, base.ids)


@pytest.mark.parametrize("n", [1, 2, 3])
def test_sensor_3d_stencils(rtod, oracle_mod, n):
    """3-d: 27 stencil cells (one round), 125 and 343 (several rounds); n >= 2
    enables the single-cell rule and, with n = 3, the neighbourhood rule."""
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    check_vs_oracle(rtod, oracle_mod, w.points, w.window, w.slide, w.R, w.K, 60, cells_per_r=n, batch=32)


@pytest.mark.parametrize("d,n", [(2, 1), (2, 2), (2, 3), (8, 1), (8, 2)])
def test_other_dims(rtod, oracle_mod, d, n):
    from rtod_b200 import datagen
    pts = datagen.random_walk(30_000, 0.1, seed=60 + d, dim=d)
    check_vs_oracle(rtod, oracle_mod, pts, 6000, 600, 0.25 * d ** 0.5, 20, 15, cells_per_r=n, batch=8)


def test_sensor_3d_sparse_and_shared_bins(rtod, oracle_mod):
    """3-d points over a range wider than the 16 x 64 x 64 bin box (bins
    shared by several cells, no pure span), with tight clusters."""
    rng = np.random.default_rng(81)
    n = 20_000
    centres = rng.uniform(-400, 400, (40, 3))
    pts = np.where(rng.random((n, 1)) < 0.7, centres[rng.integers(0, 40, n)] + rng.normal(0, 0.05, (n, 3)),
                   rng.uniform(-400, 400, (n, 3))).astype(np.float32)
    for nc in (2, 3):
        check_vs_oracle(rtod, oracle_mod, pts, 4000, 400, 0.5, 10, 30, cells_per_r=nc, batch=16)


@pytest.mark.parametrize("engine", ["span", "window"])
def test_aliased_neighbour_bin_at_range_limit(rtod, oracle_mod, engine):
    """Two clusters 65535 cells apart: the cell next to cluster A shares its
    bin with cluster B while the span's cell range is just 65536. A's points
    (fewer than K per window) are outliers; counting B's bin as A's
    neighbour cell would make them inliers."""
    R, n = 1.0, 4
    cell = R * (1 + 2.0 ** -12) / n
    kA = 30_000
    rng = np.random.default_rng(91)
    m = 12_000
    is_a = rng.random(m) < 0.2
    xa = (kA + 0.25 + 0.5 * rng.random(m)) * cell           # cell kA
    xb = (kA + 65_535 + 0.25 + 0.5 * rng.random(m)) * cell  # cell kA + 65535: bin kA - 1
    pts = np.where(is_a, xa, xb).astype(np.float32)[:, None]
    res = check_vs_oracle(rtod, oracle_mod, pts, 1000, 100, R, 300, 20, cells_per_r=n, batch=8) \
        if engine == "span" else None
    if engine == "window":
        off, ids, _ = oracle_mod.detect(pts[:1000 + 20 * 100], 1000, 100, R, 300, engine="grid", threads=8)
        r, tun = run(rtod, pts, 1000, 100, R, 300, 20, cells_per_r=n, engine="window")
        np.testing.assert_array_equal(r.offsets, off)
        np.testing.assert_array_equal(r.ids, ids)
        res = r
    # every cluster-A point of every window is an outlier
    assert res.offsets[-1] == sum(int(is_a[(j + 1) * 100:(j + 1) * 100 + 1000].sum()) for j in range(20))
