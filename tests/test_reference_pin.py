"""The oracle pinned to RTOD's own code.

tests/golden/ref_*.npz hold per-slide outlier sets produced by RTOD's host
code (src/ods/optixScan.cpp detect_outlier with its FixQueue grid filter and
outlier pick, compiled unmodified by oracle/ref/Makefile, the OptiX programs
and AABB kernel restated on the host) and confirmed slide by slide by RTOD's
brute-force check_outlier (:817-881); tests/golden/make_ref_golden.py made
them. RTOD reads and compares doubles, so the pin is the oracle's double
mode (double storage, RTOD's double predicate). Where the RTOD sources are
present, the reference build itself is re-run on a small stream as well.
"""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, golden_cases_f64, load_golden

REF_CASES = sorted(glob.glob(os.path.join(GOLDEN_DIR, "ref_*.npz")))


def load_ref(path):
    z = np.load(path)
    meta = json.loads(bytes(z["meta"]).decode())
    from rtod_b200 import datagen  # noqa: F401  (used by the stream expression)
    pts = eval(meta["stream"], {"datagen": datagen})
    pts = np.ascontiguousarray(pts, np.float32)
    if pts.ndim == 1:
        pts = pts[:, None]
    digest = hashlib.sha256(pts.tobytes()).hexdigest()[:32]
    assert digest == meta["digest"], "stream generator changed since the fixture was made"
    return meta, pts, z["offsets"], z["ids"]


def test_reference_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in REF_CASES}
    assert {"ref_walk1d_W10k", "ref_stock1d_W20k", "ref_gmm1d_W10k_K30", "ref_gmm1d_W10k_K70",
            "ref_sensor3d_W10k", "ref_sensor3d_W4k_K10"} <= names


@pytest.mark.parametrize("path", REF_CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_double_mode_matches_rtod(oracle_mod, path):
    meta, pts, off, ids = load_ref(path)
    assert meta["brute_force_agrees"] and meta["margin_events"] == 0
    assert len(off) == meta["slides"] + 1
    for engine in ("grid", "grid_nofilter"):
        o, i, _ = oracle_mod.detect(pts.astype(np.float64), meta["W"], meta["S"], meta["R"], meta["K"],
                                    "f64_lt", engine=engine, threads=8, f64=True)
        np.testing.assert_array_equal(o, off)
        np.testing.assert_array_equal(i, ids)


@pytest.mark.parametrize("path", REF_CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_float_predicate_on_rtod_streams(oracle_mod, path):
    """The FP32 predicate (the detector's default) differs from RTOD's double
    test only for pairs whose distance rounds across R; on these streams
    every slide but those with such pairs matches RTOD, and the slides that
    differ do so by points whose nearest contested neighbour sits within a
    float32 rounding of R."""
    meta, pts, off, ids = load_ref(path)
    o, i, _ = oracle_mod.detect(pts, meta["W"], meta["S"], meta["R"], meta["K"], "fp32_le", engine="grid",
                                threads=8)
    differ = [j for j in range(meta["slides"])
              if not np.array_equal(i[o[j]:o[j + 1]], ids[off[j]:off[j + 1]])]
    assert len(differ) <= max(1, meta["slides"] // 50)


def reference_available():
    try:
        from oracle import reference
    except ImportError:
        return False
    return reference.build()


@pytest.mark.skipif(not os.path.isdir("/root/reference/src/ods"), reason="RTOD sources absent")
def test_reference_build_reruns_small_streams(oracle_mod):
    """RTOD's code, rebuilt from its sources, against the oracle's double
    mode on small 1-d and 3-d streams (including the double fixtures)."""
    assert reference_available()
    from oracle import reference
    from rtod_b200 import datagen
    cases = [(datagen.random_walk(6000, 0.1, seed=21, jump_frac=0.01), 2000, 100, 0.3, 15),
             (datagen.sensor_3d(4000, seed=22), 1000, 100, 1.9, 12)]
    for path in golden_cases_f64():
        meta, pts, o, i = load_golden(path)
        if pts.shape[1] in (1, 3):
            cases.append((pts, meta["W"], meta["S"], meta["R"], meta["K"]))
    for pts, W, S, R, K in cases:
        off, ids, boff, bids, stats = reference.detect(np.asarray(pts, np.float64), W, S, R, K, brute=True)
        o, i, _ = oracle_mod.detect(np.asarray(pts, np.float64), W, S, R, K, "f64_lt", engine="grid", f64=True)
        np.testing.assert_array_equal(o, off)
        np.testing.assert_array_equal(i, ids)
        if stats[1] == 0:
            np.testing.assert_array_equal(boff, off)
            np.testing.assert_array_equal(bids, ids)
