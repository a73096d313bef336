"""The CPU oracle against the golden fixtures and against itself (CPU only)."""
import os

import numpy as np
import pytest

from conftest import golden_cases, golden_cases_f64, load_golden


@pytest.mark.parametrize("path", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("engine", ["brute", "grid", "grid_nofilter"])
def test_oracle_matches_golden(oracle_mod, path, engine):
    meta, pts, off, ids = load_golden(path)
    o, i, _ = oracle_mod.detect(pts, meta["W"], meta["S"], meta["R"], meta["K"], meta["pred"],
                                engine=engine)
    np.testing.assert_array_equal(o, off)
    np.testing.assert_array_equal(i, ids)


@pytest.mark.parametrize("path", golden_cases_f64(), ids=lambda p: os.path.basename(p)[:-4])
@pytest.mark.parametrize("engine", ["brute", "grid", "grid_nofilter"])
def test_oracle_double_storage_matches_golden(oracle_mod, path, engine):
    meta, pts, off, ids = load_golden(path)
    assert pts.dtype == np.float64 and meta["coord"] == "f64"
    o, i, _ = oracle_mod.detect(pts, meta["W"], meta["S"], meta["R"], meta["K"], "f64_lt", engine=engine,
                                f64=True)
    np.testing.assert_array_equal(o, off)
    np.testing.assert_array_equal(i, ids)


def test_oracle_double_storage_differs_from_float_storage(oracle_mod):
    """The pair 1e-12 inside R: neighbours as doubles, not once rounded to float32."""
    assert oracle_mod.pred_f64([0.0], [0.1 - 1e-12], 0.1)
    assert not oracle_mod.pred(np.float32([0.0]), np.float32([0.1 - 1e-12]), 0.1, "f64_lt")


def test_oracle_threads_agree(oracle_mod):
    from rtod_b200 import datagen
    pts = datagen.random_walk(40_000, 0.1, seed=5, jump_frac=0.005)
    a = oracle_mod.detect(pts, 4000, 200, 0.3, 20, engine="grid", threads=1)
    b = oracle_mod.detect(pts, 4000, 200, 0.3, 20, engine="grid", threads=4)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_oracle_grid_vs_brute_3d(oracle_mod):
    from rtod_b200 import datagen
    pts = datagen.sensor_3d(6000, seed=21)
    for pred in ("fp32_le", "f64_lt"):
        a = oracle_mod.detect(pts, 2000, 500, 1.9, 4, pred, engine="brute")
        b = oracle_mod.detect(pts, 2000, 500, 1.9, 4, pred, engine="grid")
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
        # the grid filter must skip most of the dense sensor points
        assert b[2][0] < a[2][0]


def test_oracle_predicate_known_answers(oracle_mod):
    f = np.float32
    assert oracle_mod.pred([0.0], [0.5], 0.5, "fp32_le")
    assert not oracle_mod.pred([0.0], [0.5], 0.5, "f64_lt")
    assert not oracle_mod.pred([0.0], [np.nextafter(f(0.5), f(1))], 0.5, "fp32_le")
    assert oracle_mod.pred([0.0], [np.nextafter(f(0.5), f(0))], 0.5, "f64_lt")
    assert oracle_mod.pred([0, 0, 0], [0.25, 0.25, 0.25], 0.5, "fp32_le")
    assert not oracle_mod.pred([0, 0, 0], [0.5, 0.25, 0], 0.5, "fp32_le")


def test_oracle_rejects_bad_config(oracle_mod):
    pts = np.zeros(10, np.float32)
    with pytest.raises(ValueError):
        oracle_mod.detect(pts, 4, 3, 1.0, 1)  # W % S != 0
    bad = pts.copy()
    bad[3] = np.nan
    with pytest.raises(ValueError):
        oracle_mod.detect(bad, 4, 2, 1.0, 1)
