"""Batched streams (many uneven streams advanced together, one graph replay
per step) against the CPU oracle, stream by stream, slide by slide."""
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


def make_streams(n=9, seed=5, slides=12):
    from rtod_b200 import datagen
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        d = [1, 3, 8][i % 3]
        W = int(rng.choice([2000, 3000, 5000, 8000]))
        S = W // int(rng.choice([4, 10, 20]))
        if rng.random() < 0.5:
            pts = datagen.random_walk(W + slides * S, 0.1, seed=100 + i, dim=d)
        else:
            pts = datagen.gaussian_mixture(W + slides * S, seed=100 + i, dim=d)
        R = {1: 0.05, 3: 0.3, 8: 0.6}[d] if i % 2 else {1: 0.02, 3: 0.2, 8: 0.5}[d]
        out.append(dict(window=W, slide=S, R=R, K=10 + i, dim=d, points=pts, slides=slides,
                        pred="f64_lt" if i == 4 else "fp32_le"))
    return out


@pytest.mark.parametrize("router,count,pipeline", [(False, "auto", "fused"), (True, "auto", "fused"),
                                                   (False, "group", "fused"), (True, "point", "fused"),
                                                   (False, "auto", "staged"), (True, "auto", "staged"),
                                                   (True, "group8", "staged")])
def test_batch_matches_oracle(rtod, oracle_mod, router, count, pipeline):
    """count "group8": the 8-d streams on group counts (unrouted, a branch of
    the step's graph of their own) beside the routed groups (one branch)."""
    streams = make_streams()
    expect = []
    for st in streams:
        off, ids, _ = oracle_mod.detect(st["points"], st["window"], st["slide"], st["R"], st["K"],
                                        st["pred"], engine="grid", threads=4)
        expect.append((off, ids))
    cfg = [dict({k: st[k] for k in ("window", "slide", "R", "K", "dim", "pred")},
                count=("group" if st["dim"] == 8 else "auto") if count == "group8" else count, pipeline=pipeline)
           for st in streams]
    with rtod.BatchDetector(cfg, router=router) as bd:
        for i, st in enumerate(streams):
            bd.push(i, st["points"][:st["window"]])
        done = [0] * len(streams)
        for step in range(40):
            for i, st in enumerate(streams):
                # stream 2 sits out every third step; all stop after their slides
                if done[i] < st["slides"] and not (i == 2 and step % 3 == 1):
                    W, S = st["window"], st["slide"]
                    bd.push(i, st["points"][W + done[i] * S:W + (done[i] + 1) * S])
            pushed = [done[i] < st["slides"] and not (i == 2 and step % 3 == 1)
                      for i, st in enumerate(streams)]
            if not any(pushed):
                continue
            res = bd.step()
            for i, st in enumerate(streams):
                if pushed[i]:
                    off, ids = expect[i]
                    j = done[i]
                    np.testing.assert_array_equal(res[i], ids[off[j]:off[j + 1]])
                    done[i] += 1
                else:
                    assert res[i].size == 0
        assert all(done[i] == st["slides"] for i, st in enumerate(streams))
        stats = bd.stats
        assert stats["groups"] == 4  # d=1, d=3, d=8 with fp32, and the f64 stream
        assert stats["pair_tests"] >= 0
        assert stats["detections"] == sum(st["slides"] for st in streams)


def test_batch_push_buffer_reused_at_once(rtod, oracle_mod):
    """Slides pushed from one page-locked buffer that the caller overwrites
    right after each push: every step still detects the pushed points."""
    import torch
    streams = make_streams(n=3, seed=7)
    expect = [oracle_mod.detect(st["points"], st["window"], st["slide"], st["R"], st["K"], st["pred"],
                                engine="grid", threads=4)[:2] for st in streams]
    cfg = [{k: st[k] for k in ("window", "slide", "R", "K", "dim", "pred")} for st in streams]
    bufs = [torch.empty((st["slide"], st["dim"]), dtype=torch.float32).pin_memory() for st in streams]
    with rtod.BatchDetector(cfg) as bd:
        for i, st in enumerate(streams):
            bd.push(i, st["points"][:st["window"]])
        for j in range(min(st["slides"] for st in streams)):
            for i, st in enumerate(streams):
                W, S = st["window"], st["slide"]
                bufs[i].copy_(torch.from_numpy(st["points"][W + j * S:W + (j + 1) * S]))
                bd.push(i, bufs[i].numpy())
                bufs[i].fill_(1e30)
            res = bd.step()
            for i in range(len(streams)):
                off, ids = expect[i]
                np.testing.assert_array_equal(res[i], ids[off[j]:off[j + 1]])


@pytest.mark.parametrize("router", [False, True])
def test_batch_autotuner_keeps_results(rtod, oracle_mod, router):
    """With the autotuner on, the first steps try every group's candidate
    settings (cell width with the rings re-keyed, count block shape, count
    mode beyond 3-d), one per step; every step's outliers still match the
    oracle, and every group settles on one setting."""
    streams = make_streams(n=6, seed=9, slides=30)
    expect = [oracle_mod.detect(st["points"], st["window"], st["slide"], st["R"], st["K"], st["pred"],
                                engine="grid", threads=4)[:2] for st in streams]
    cfg = [{k: st[k] for k in ("window", "slide", "R", "K", "dim", "pred")} for st in streams]
    with rtod.BatchDetector(cfg, router=router, tuner=True) as bd:
        before = bd.tuning
        assert not all(g["settled"] for g in before)
        for i, st in enumerate(streams):
            bd.push(i, st["points"][:st["window"]])
        seen = {}
        for j in range(30):
            for i, st in enumerate(streams):
                W, S = st["window"], st["slide"]
                bd.push(i, st["points"][W + j * S:W + (j + 1) * S])
            res = bd.step()
            for g in bd.tuning:
                seen.setdefault((g["dim"], g["pred"]), set()).add((g["cells_per_r"], g["block_warps"], g["count"]))
            for i in range(len(streams)):
                off, ids = expect[i]
                np.testing.assert_array_equal(res[i], ids[off[j]:off[j + 1]], err_msg=f"stream {i} slide {j}")
        after = bd.tuning
        assert all(g["settled"] for g in after)
        assert all(len(v) > 1 for v in seen.values())  # each group tried several settings


@pytest.mark.parametrize("dim,count", [(1, "point"), (8, "group")])
def test_batch_more_streams_of_one_kind_than_one_launch_holds(rtod, oracle_mod, dim, count):
    """260 streams of one (dimension, predicate, count mode): a launch's
    count list holds at most 256 jobs, so they run as two groups. Every
    stream is checked against the oracle slide by slide; every seventh
    stream sits one step out."""
    from rtod_b200 import datagen
    n, W, S, slides, K = 260, 400, 40, 3, 5
    R = 0.05 if dim == 1 else 0.5
    streams = [datagen.random_walk(W + slides * S, 0.1, seed=3000 + i, dim=dim) for i in range(n)]
    expect = [oracle_mod.detect(p, W, S, R, K, "fp32_le", engine="grid", threads=4)[:2] for p in streams]
    cfg = [dict(window=W, slide=S, R=R, K=K, dim=dim, count=count) for _ in range(n)]
    with rtod.BatchDetector(cfg) as bd:
        for i, p in enumerate(streams):
            bd.push(i, p[:W])
        done = [0] * n
        for step in range(slides + 1):
            pushed = [done[i] < slides and not (i % 7 == 3 and step == 1) for i in range(n)]
            for i, p in enumerate(streams):
                if pushed[i]:
                    bd.push(i, p[W + done[i] * S:W + (done[i] + 1) * S])
            res = bd.step()
            for i in range(n):
                if pushed[i]:
                    off, ids = expect[i]
                    j = done[i]
                    np.testing.assert_array_equal(res[i], ids[off[j]:off[j + 1]])
                    done[i] += 1
                else:
                    assert res[i].size == 0
        assert done == [slides] * n
        assert bd.stats["groups"] == 2
