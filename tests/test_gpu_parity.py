"""GPU parity: the CUDA path, called through the C ABI, against the golden
fixtures and the CPU oracle. Bit-exact: the per-slide outlier ID sets must be
identical."""
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
@pytest.mark.parametrize("opt,graph,n", [(2, True, 0), (0, False, 0), (2, False, 1), (1, True, 3)])
@pytest.mark.parametrize("engine", ["window", "span"])
def test_run_matches_golden(rtod, path, opt, graph, n, engine):
    meta, pts, off, ids = load_golden(path)
    with rtod.Detector(meta["W"], meta["S"], meta["R"], meta["K"], dim=pts.shape[1], opt=opt,
                       pred=meta["pred"], use_graph=graph, cells_per_r=n, engine=engine) as det:
        assert_same(det.run(pts), off, ids)
        assert det.tuning["engine"] == engine


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("pipeline,graph", [("fused", True), ("fused", False), ("staged", True)])
def test_push_detect_matches_golden(rtod, path, pipeline, graph):
    """RTOD's per-slide loop: push S points, detect; the fused pipeline (one
    cooperative launch per detection) and the staged one."""
    meta, pts, off, ids = load_golden(path)
    W, S = meta["W"], meta["S"]
    with rtod.Detector(W, S, meta["R"], meta["K"], dim=pts.shape[1], pred=meta["pred"], pipeline=pipeline,
                       use_graph=graph) as det:
        det.push(pts[:W])
        for j in range(len(off) - 1):
            det.push(pts[W + j * S:W + (j + 1) * S])
            got = det.detect()
            np.testing.assert_array_equal(got, ids[off[j]:off[j + 1]])
        assert det.slides_done == len(off) - 1


@pytest.mark.parametrize("kw", [dict(), dict(router=True), dict(count="group"), dict(cells_per_r=4),
                                dict(pred="f64_lt"), dict(router=True, use_graph=False),
                                dict(pipeline="fused"), dict(pipeline="fused", router=True)])
def test_push_detect_stock_like_stream(rtod, oracle_mod, kw):
    """The stock-like stream (W=100k, S=5k) slide by slide, 40 slides, against
    the oracle; every seventh detection asks for stage times (the staged
    pipeline then runs, with per-stage events) and must agree too."""
    from rtod_b200 import datagen
    w = datagen.stock_like()
    n = 40
    pred = kw.get("pred", "fp32_le")
    off, ids, _ = oracle_mod.detect(w.points[:w.window + n * w.slide], w.window, w.slide, w.R, w.K, pred,
                                    engine="grid", threads=os.cpu_count() or 4)
    with rtod.Detector(w.window, w.slide, w.R, w.K, **kw) as det:
        det.push(w.points[:w.window])
        for j in range(n):
            det.push(w.points[w.window + j * w.slide:w.window + (j + 1) * w.slide])
            got = det.detect(times=(j % 7 == 3))
            if isinstance(got, tuple):
                got = got[0]
            np.testing.assert_array_equal(got, ids[off[j]:off[j + 1]])


@pytest.mark.parametrize("source", ["host", "pinned", "device"])
def test_push_buffer_reused_at_once(rtod, source):
    """The caller may overwrite a pushed slide's buffer right after the push
    returns: the detection still sees the pushed points (host slides are
    copied into a page-locked buffer during the push)."""
    import torch
    meta, pts, off, ids = load_golden(golden_cases()[-1])
    W, S = meta["W"], meta["S"]
    buf = torch.empty((S, pts.shape[1]), dtype=torch.float32)
    if source == "pinned":
        buf = buf.pin_memory()
    if source == "device":
        buf = buf.cuda()
    with rtod.Detector(W, S, meta["R"], meta["K"], dim=pts.shape[1], pred=meta["pred"]) as det:
        det.push(pts[:W])
        for j in range(len(off) - 1):
            buf.copy_(torch.from_numpy(pts[W + j * S:W + (j + 1) * S]))
            det.push(buf.numpy() if source != "device" else buf)
            buf.fill_(1e30)  # garbage: must not reach the detection
            np.testing.assert_array_equal(det.detect(), ids[off[j]:off[j + 1]])


def oracle_check(rtod, oracle_mod, pts, W, S, R, K, slides, pred="fp32_le", **kw):
    pts = pts[:W + slides * S]
    off, ids, _ = oracle_mod.detect(pts, W, S, R, K, pred, engine="grid", threads=os.cpu_count() or 4)
    with rtod.Detector(W, S, R, K, dim=pts.shape[1] if pts.ndim == 2 else 1, pred=pred, **kw) as det:
        r = det.run(pts)
        assert r.slides == slides
        assert_same(r, off, ids)
    return off, ids


def test_small_walk_full_stream(rtod, oracle_mod):
    from rtod_b200 import datagen
    w = datagen.small_walk()
    oracle_check(rtod, oracle_mod, w.points, w.window, w.slide, w.R, w.K, w.slides)


@pytest.mark.parametrize("kw", [dict(), dict(engine="window"), dict(tuner=True, router=True)])
def test_stock_like_full_stream(rtod, oracle_mod, kw):
    """Every slide (189) of the stock-like stream, W=100k, S=5k."""
    from rtod_b200 import datagen
    w = datagen.stock_like()
    off, _ = oracle_check(rtod, oracle_mod, w.points, w.window, w.slide, w.R, w.K, w.slides, **kw)
    assert len(off) == 190


@pytest.mark.parametrize("pred,kw", [("fp32_le", dict()), ("fp32_le", dict(engine="window", router=True)),
                                     ("f64_lt", dict())])
def test_sensor_like_full_stream(rtod, oracle_mod, pred, kw):
    """Every slide (1130) of the 3-d sensor-like stream, W=10k, S=500,
    under both predicates; the router on the window engine."""
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    oracle_check(rtod, oracle_mod, w.points, w.window, w.slide, w.R, w.K, w.slides, pred=pred, **kw)


@pytest.mark.parametrize("K", [30, 50, 70])
def test_gaussian_like_K_sweep(rtod, oracle_mod, K):
    """Every slide (180) of the Gaussian-mixture stream for each K."""
    from rtod_b200 import datagen
    w = datagen.gaussian_like(K)
    oracle_check(rtod, oracle_mod, w.points, w.window, w.slide, w.R, w.K, w.slides)
    oracle_check(rtod, oracle_mod, w.points, w.window, w.slide, w.R, w.K, w.slides, engine="window", router=True)


@pytest.fixture(scope="module")
def batched_expect(oracle_mod):
    """The 64 uneven streams of the batched workload (W log-uniform in
    [5k, 200k], S = W/20, d in {1, 3, 8}) and the oracle's outliers of their
    first 3 slides."""
    from rtod_b200 import datagen
    streams = datagen.batched_streams(slides=3)
    expect = [oracle_mod.detect(w.points, w.window, w.slide, w.R, w.K, engine="grid",
                                threads=os.cpu_count() or 4)[:2] for w in streams]
    return streams, expect


@pytest.mark.parametrize("router,pipeline", [(False, "fused"), (True, "fused"), (False, "staged")])
def test_batched_streams_first_slides(rtod, batched_expect, router, pipeline):
    """All 64 streams of the batched workload through the multi-stream API
    (one graph replay per step), first 3 slides of every stream."""
    streams, expect = batched_expect
    cfg = [dict(window=w.window, slide=w.slide, R=w.R, K=w.K, dim=w.dim, pipeline=pipeline) for w in streams]
    with rtod.BatchDetector(cfg, router=router) as bd:
        for i, w in enumerate(streams):
            bd.push(i, w.points[:w.window])
        for j in range(3):
            for i, w in enumerate(streams):
                bd.push(i, w.points[w.window + j * w.slide:w.window + (j + 1) * w.slide])
            res = bd.step()
            for i in range(len(streams)):
                off, ids = expect[i]
                np.testing.assert_array_equal(res[i], ids[off[j]:off[j + 1]], err_msg=streams[i].name)


def test_batched_streams_span_engine(rtod, batched_expect):
    """The same 64 streams, each through rtod_run (tuned engine), first 3 slides."""
    streams, expect = batched_expect
    for w, (off, ids) in zip(streams, expect):
        with rtod.Detector(w.window, w.slide, w.R, w.K, dim=w.dim) as det:
            assert_same(det.run(w.points), off, ids)


@pytest.mark.parametrize("d", [2, 5, 8])
def test_higher_dims(rtod, oracle_mod, d):
    from rtod_b200 import datagen
    pts = datagen.random_walk(30_000, 0.1, seed=40 + d, dim=d)
    oracle_check(rtod, oracle_mod, pts, 6000, 600, 0.25 * d ** 0.5, 20, 15)


def test_full_size_properties(rtod):
    """Full stock-like stream (189 slides): every configuration of the grid
    and launch gives the same outlier sets, IDs are sorted and in-window."""
    from rtod_b200 import datagen
    w = datagen.stock_like()
    runs = []
    for kw in (dict(engine="window"), dict(opt=0), dict(cells_per_r=1), dict(cells_per_r=3, use_graph=False),
               dict(block_warps=2), dict(cells_per_r=4), dict(cells_per_r=7, batch=5),
               dict(engine="window", cells_per_r=4), dict(engine="window", cells_per_r=7, batch=5),
               dict(engine="span", batch=64), dict(engine="span", batch=1), dict(engine="span", opt=0, batch=13)):
        with rtod.Detector(w.window, w.slide, w.R, w.K, **kw) as det:
            runs.append(det.run(w.points))
    base = runs[0]
    assert base.slides == w.slides
    for r in runs[1:]:
        assert_same(r, base.offsets, base.ids)
    for j in range(base.slides):
        s = base.slide(j)
        lo = (j + 1) * w.slide
        assert np.all(np.diff(s) > 0)
        assert s.size == 0 or (s[0] >= lo and s[-1] < lo + w.window)


def test_device_pointers(rtod):
    import torch
    meta, pts, off, ids = load_golden(golden_cases()[-1])
    dev = torch.from_numpy(pts).cuda()
    out = torch.empty(max(1, len(ids)) + 16, dtype=torch.int64, device="cuda")
    with rtod.Detector(meta["W"], meta["S"], meta["R"], meta["K"], dim=pts.shape[1],
                       pred=meta["pred"]) as det:
        r = det.run(dev, out_ids=out, ids_cap=out.numel())
        np.testing.assert_array_equal(r.offsets, off)
        np.testing.assert_array_equal(r.ids.cpu().numpy(), ids)


def test_output_buffers(rtod):
    """IDs into pageable host memory (one copy after the pass), page-locked
    host memory (written during the pass through its device mapping) and
    device memory; replays with another page-locked buffer; a capacity error
    writes nothing past the capacity."""
    import torch
    from rtod_b200 import datagen
    w = datagen.stock_like()
    pts = w.points[:w.window + 40 * w.slide]
    with rtod.Detector(w.window, w.slide, w.R, w.K, engine="span") as det:
        ref = det.run(pts)
        n = len(ref.ids)
        for _ in range(2):
            for pinned in (True, False):
                buf = torch.full((n + 64,), -7, dtype=torch.int64)
                if pinned:
                    buf = buf.pin_memory()
                det.reset()
                r = det.run(pts, out_ids=buf.numpy(), ids_cap=n + 64)
                np.testing.assert_array_equal(r.offsets, ref.offsets)
                np.testing.assert_array_equal(buf.numpy()[:n], ref.ids)
                assert np.all(buf.numpy()[n:] == -7)
        dev = torch.full((n,), -7, dtype=torch.int64, device="cuda")
        det.reset()
        r = det.run(torch.from_numpy(pts).cuda(), out_ids=dev, ids_cap=n)
        np.testing.assert_array_equal(dev.cpu().numpy(), ref.ids)
        small = torch.full((n,), -7, dtype=torch.int64).pin_memory()
        det.reset()
        with pytest.raises(rtod.RtodError):
            det.run(pts, out_ids=small.numpy(), ids_cap=n // 2)
        assert np.all(small.numpy()[n // 2:] == -7)


@pytest.mark.parametrize("kw", [dict(engine="span"), dict(engine="span", batch=16), dict(engine="span", batch=1),
                                dict(engine="span", use_graph=False), dict(engine="window")])
def test_page_locked_input(rtod, kw):
    """A page-locked host stream: copied in pieces on a second stream, the
    first piece in parts followed by the histogram part by part (run graph of
    the span engine); the same results as from device memory, replay after
    replay."""
    import torch
    from rtod_b200 import datagen
    w = datagen.stock_like()
    pts = torch.from_numpy(w.points).pin_memory()
    with rtod.Detector(w.window, w.slide, w.R, w.K, **kw) as det:
        ref = det.run(pts.cuda())
        for _ in range(3):
            det.reset()
            assert_same(det.run(pts.numpy()), ref.offsets, ref.ids)
        det.reset()
        part = pts[:(w.window + 37 * w.slide)]  # a shorter stream: another graph
        r = det.run(part.numpy())
        assert_same(r, ref.offsets[:38], ref.ids[:ref.offsets[37]])


def test_input_errors(rtod):
    pts = np.zeros(40, np.float32)
    pts[25] = np.nan
    with rtod.Detector(10, 5, 1.0, 2) as det:
        with pytest.raises(rtod.RtodError, match="INPUT"):
            det.run(pts)
        det.reset()
        det.run(np.zeros(40, np.float32))
    big = np.zeros(40, np.float32)
    big[30] = 3e30
    with rtod.Detector(10, 5, 1e-6, 2) as det:
        with pytest.raises(rtod.RtodError, match="INPUT"):
            det.run(big)
    with rtod.Detector(10, 5, 1.0, 2) as det:
        with pytest.raises(rtod.RtodError, match="STATE"):
            det.push(np.zeros(5, np.float32))  # first push must be W points
        det.push(np.zeros(10, np.float32))
        with pytest.raises(rtod.RtodError, match="STATE"):
            det.detect()
        det.push(np.zeros(5, np.float32))
        with pytest.raises(rtod.RtodError, match="STATE"):
            det.push(np.zeros(5, np.float32))  # detect must come first
        assert det.detect().size == 0


@pytest.mark.parametrize("router", [False, True])
def test_autotuner_keeps_results(rtod, router):
    """The autotuner only changes speed: tuned and default runs agree, and the
    chosen settings are among the candidates."""
    from rtod_b200 import datagen
    w = datagen.sensor_like()
    pts = w.points[:w.window + 150 * w.slide]
    with rtod.Detector(w.window, w.slide, w.R, w.K, dim=3) as base, \
            rtod.Detector(w.window, w.slide, w.R, w.K, dim=3, tuner=True, router=router) as tuned:
        a = base.run(pts)
        b = tuned.run(pts)
        assert_same(b, a.offsets, a.ids)
        t = tuned.tuning
        assert t["cells_per_r"] in (1, 2, 3) and t["block_warps"] in (2, 4, 8)
        assert t["batch"] in (8, 16, 32, 64, 128, 256) and t["engine"] in ("span", "window")
        tuned.reset()
        assert_same(tuned.run(pts), a.offsets, a.ids)


@pytest.mark.parametrize("path", [p for p in golden_cases() if load_golden(p)[1].shape[1] == 1],
                         ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("n", [4, 6, 8])
def test_fine_cells_1d_match_golden(rtod, path, n):
    """1-d grids of R/n cells: the group filter (runs of n-1 cells) and the
    wider stencil give the same outliers."""
    meta, pts, off, ids = load_golden(path)
    with rtod.Detector(meta["W"], meta["S"], meta["R"], meta["K"], pred=meta["pred"],
                       cells_per_r=n) as det:
        assert_same(det.run(pts), off, ids)


def test_handles_on_several_host_threads(rtod):
    """One handle per host thread, all running at once (each handle owns its
    stream and graphs; the tuner's cache is shared): the same results as one
    after another."""
    import threading
    from rtod_b200 import datagen
    cases = [datagen.small_walk(), datagen.sensor_like(), datagen.gaussian_like(30), datagen.small_walk()]
    def run(w, tuner):
        with rtod.Detector(w.window, w.slide, w.R, w.K, dim=w.dim, tuner=tuner) as det:
            return det.run(w.points, max_slides=40)
    ref = [run(w, False) for w in cases]
    got = [None] * len(cases)
    errs = []
    def worker(i):
        try:
            for _ in range(3):
                got[i] = run(cases[i], i % 2 == 1)
        except Exception as e:  # surfaced below
            errs.append(e)
    th = [threading.Thread(target=worker, args=(i,)) for i in range(len(cases))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for r, g in zip(ref, got):
        assert_same(g, r.offsets, r.ids)
