"""The learned router: its network against the double-precision CPU
restatement (forward, gradient, Adam step), and the detector with the router
on against the detector with it off (identical outliers; training reduces the
loss and the misroute rate)."""
import numpy as np
import pytest


def random_params(rng, P):
    return (rng.standard_normal(P) * 0.3).astype(np.float32)


def sample_batch(rng, n):
    x = np.stack([rng.uniform(0, 1, n), rng.uniform(0, 1.2, n), rng.uniform(-1, 2, n)], 1).astype(np.float32)
    y = rng.integers(0, 4, n).astype(np.int32)
    return x, y


# ---------------------------------------------------------------------------
# CPU: the oracle's gradient against central finite differences (double).
# ---------------------------------------------------------------------------
def test_oracle_gradient_matches_finite_differences(oracle_mod):
    rng = np.random.default_rng(0)
    P = oracle_mod.mlp_param_count()
    params = random_params(rng, P)
    x, y = sample_batch(rng, 37)
    loss, g = oracle_mod.mlp_loss_grad(params, x, y)
    idx = rng.choice(P, 60, replace=False)
    eps = 1e-3
    for i in idx:
        pp, pm = params.astype(np.float64).copy(), params.astype(np.float64).copy()
        pp[i] += eps
        pm[i] -= eps
        # parameters are float32 in the oracle; use steps representable in float32
        lp, _ = oracle_mod.mlp_loss_grad(pp.astype(np.float32), x, y)
        lm, _ = oracle_mod.mlp_loss_grad(pm.astype(np.float32), x, y)
        h = float(np.float32(pp[i]) - np.float32(pm[i]))
        fd = (lp - lm) / h
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(g[i])), (i, fd, g[i])


# ---------------------------------------------------------------------------
# GPU: the CUDA forward / backward / Adam kernels against the oracle.
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rtod_b200 import build
    build.build()
    import rtod_b200
    from rtod_b200 import mlp
    return rtod_b200, mlp


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 50, 128, 300])
def test_gpu_forward_and_gradient_match_oracle(gpu, oracle_mod, n):
    _, mlp = gpu
    rng = np.random.default_rng(n)
    P = mlp.param_count()
    assert P == oracle_mod.mlp_param_count()
    params = random_params(rng, P)
    x, y = sample_batch(rng, n)
    z = mlp.forward(params, x)
    zref = oracle_mod.mlp_forward(params, x)
    np.testing.assert_allclose(z, zref, rtol=1e-4, atol=1e-4)  # FP32 vs double
    loss, g = mlp.loss_grad(params, x, y)
    lref, gref = oracle_mod.mlp_loss_grad(params, x, y)
    assert abs(loss - lref) <= 1e-4 * max(1.0, abs(lref))
    np.testing.assert_allclose(g, gref, rtol=1e-3, atol=2e-5)


@pytest.mark.gpu
def test_gpu_adam_step_matches_oracle(gpu, oracle_mod):
    _, mlp = gpu
    rng = np.random.default_rng(7)
    P = mlp.param_count()
    params = random_params(rng, P)
    m = (rng.standard_normal(P) * 1e-3).astype(np.float32)
    v = (rng.random(P) * 1e-5).astype(np.float32)
    x, y = sample_batch(rng, 200)
    t = 5
    p1, m1, v1, _ = mlp.adam_step(params, m, v, t, x, y, lr=1e-3)
    _, gref = oracle_mod.mlp_loss_grad(params, x, y)
    p2, m2, v2 = oracle_mod.mlp_adam(params, m, v, gref.astype(np.float32), t)
    np.testing.assert_allclose(m1, m2, rtol=2e-3, atol=1e-7)
    np.testing.assert_allclose(v1, v2, rtol=2e-3, atol=1e-10)
    np.testing.assert_allclose(p1, p2, rtol=1e-5, atol=2e-6)


@pytest.mark.gpu
def test_gpu_training_reduces_loss(gpu, oracle_mod):
    _, mlp = gpu
    rng = np.random.default_rng(3)
    P = mlp.param_count()
    params = random_params(rng, P) * 0.3
    x = rng.uniform(0, 1, (256, 3)).astype(np.float32)
    y = (x[:, 0] * 3.99).astype(np.int32)  # a learnable rule
    m = np.zeros(P, np.float32)
    v = np.zeros(P, np.float32)
    l0, _ = oracle_mod.mlp_loss_grad(params, x, y)
    for t in range(1, 201):
        params, m, v, _ = mlp.adam_step(params, m, v, t, x, y, lr=1e-2)
    l1, _ = oracle_mod.mlp_loss_grad(params, x, y)
    assert l1 < 0.5 * l0


# ---------------------------------------------------------------------------
# GPU: router on vs off.
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("case", ["stk", "tao", "gau", "walk8"])
def test_router_results_identical_to_plain(gpu, oracle_mod, case):
    rtod, _ = gpu
    from rtod_b200 import datagen
    if case == "stk":
        w = datagen.stock_like()
        pts, W, S, R, K, sl = w.points, w.window, w.slide, w.R, w.K, 40
    elif case == "tao":
        w = datagen.sensor_like()
        pts, W, S, R, K, sl = w.points, w.window, w.slide, w.R, w.K, 200
    elif case == "gau":
        w = datagen.gaussian_like(30)
        pts, W, S, R, K, sl = w.points, w.window, w.slide, w.R, w.K, 30
    else:
        pts = datagen.random_walk(40_000, 0.1, seed=9, dim=8)
        W, S, R, K, sl = 8000, 400, 0.6, 20, 40
    dim = pts.shape[1]
    # the span engine routes where its stencils have at most 32 cells (3-d:
    # one cell per R) and up to 3 dimensions; the 8-d stream is routed by the
    # window engine's point queues
    kw = dict(cells_per_r=1) if case == "tao" else (dict(engine="window", count="point") if case == "walk8" else {})
    with rtod.Detector(W, S, R, K, dim=dim, router=False, **kw) as plain, \
            rtod.Detector(W, S, R, K, dim=dim, router=True, **kw) as routed:
        a = plain.run(pts, max_slides=sl)
        for _ in range(3):  # the router keeps training across runs
            routed.reset()
            b = routed.run(pts, max_slides=sl)
            np.testing.assert_array_equal(a.offsets, b.offsets)
            np.testing.assert_array_equal(a.ids, b.ids)
        info = routed.router_info()
        assert info["steps"] > 0
        assert info["routed_early"] + info["routed_sweep"] > 0
    if case == "tao":
        off, ids, _ = oracle_mod.detect(pts[:W + sl * S], W, S, R, K, engine="grid", threads=8)
        np.testing.assert_array_equal(a.offsets, off)
        np.testing.assert_array_equal(a.ids, ids)


@pytest.mark.gpu
def test_router_learns_to_spot_outliers(gpu):
    """On the Gaussian-mixture stream most counted points are outliers (noise
    between the clusters): the untrained network (biased towards inliers)
    sends them all to the early-exit queue, the trained one routes them to
    the full-sweep queue and misroutes far fewer points. Results are the
    same either way."""
    rtod, _ = gpu
    from rtod_b200 import datagen
    w = datagen.gaussian_like(30)
    with rtod.Detector(w.window, w.slide, w.R, w.K, engine="window") as plain:
        ref = plain.run(w.points, max_slides=64)
    with rtod.Detector(w.window, w.slide, w.R, w.K, engine="window", router=True) as det:
        r = det.run(w.points, max_slides=64)
        i0 = det.router_info()
        first = i0["misrouted"] / max(1, i0["routed_early"] + i0["routed_sweep"])
        for _ in range(8):
            det.reset()
            r = det.run(w.points, max_slides=64)
        i1 = det.router_info()
        n = i1["routed_early"] + i1["routed_sweep"] - i0["routed_early"] - i0["routed_sweep"]
        later = (i1["misrouted"] - i0["misrouted"]) / max(1, n)
        sweep = (i1["routed_sweep"] - i0["routed_sweep"]) / max(1, n)
    np.testing.assert_array_equal(r.offsets, ref.offsets)
    np.testing.assert_array_equal(r.ids, ref.ids)
    assert first > 0.5            # untrained: the outliers go to the early-exit queue
    assert later < 0.5 * first    # trained: far fewer misroutes
    assert sweep > 0.3            # the outliers now take the full-sweep queue


@pytest.mark.gpu
def test_trained_router_beats_untrained(gpu):
    """What the trained network gains, on the sensor-like 3-d stream (span
    engine, one cell per R, where most runs cost less in delta segments):
    untrained (biased towards independent counts) it sends almost nothing
    to delta segments, trained most runs; and the trained routing runs the
    pass faster than the same engine with the router off (median device
    time of 9 passes), with identical outliers."""
    rtod, _ = gpu
    import torch
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    pts = torch.from_numpy(w.points).cuda()
    out = torch.empty(w.slides * w.window // 4, dtype=torch.int64, device="cuda")

    def timed(det):
        ts = []
        for _ in range(9):
            det.reset()
            r = det.run(pts, out_ids=out, ids_cap=out.numel(), times=True)
            ts.append(r.times["total"])
        return float(np.median(ts)), r.offsets.copy(), out[:int(r.offsets[-1])].cpu().numpy()

    with rtod.Detector(w.window, w.slide, w.R, w.K, dim=3, engine="span", cells_per_r=1, batch=256) as plain:
        t_plain, off, ids = timed(plain)
    with rtod.Detector(w.window, w.slide, w.R, w.K, dim=3, engine="span", cells_per_r=1, batch=256,
                       router=True) as det:
        det.run(pts, out_ids=out, ids_cap=out.numel())
        i0 = det.router_info()
        first = i0["routed_sweep"] / max(1, i0["routed_early"] + i0["routed_sweep"])
        for _ in range(30):
            det.reset()
            det.run(pts, out_ids=out, ids_cap=out.numel())
        i1 = det.router_info()
        t_routed, off2, ids2 = timed(det)
        i2 = det.router_info()
        later = (i2["routed_sweep"] - i1["routed_sweep"]) / max(
            1, i2["routed_early"] + i2["routed_sweep"] - i1["routed_early"] - i1["routed_sweep"])
    np.testing.assert_array_equal(off2, off)
    np.testing.assert_array_equal(ids2, ids)
    assert i1["steps"] > i0["steps"]
    assert first < 0.2 and later > 0.5
    assert t_routed < 0.96 * t_plain, (t_routed, t_plain)
