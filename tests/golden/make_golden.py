"""Generates the golden fixtures in this folder.

RTOD has no tests, golden vectors or data files, and its detector needs
OptiX and RT cores, so it cannot be run to produce reference outputs. The
fixtures are therefore produced here by an independent numpy brute force of
the detection rule (count of window points within R, self included; outlier
iff count <= K; src/ods/optixScan.cu:158-199, src/ods/optixScan.cpp:817-881,
slide schedule src/ods/optixScan.cpp:1036-1108), plus known-answer cases whose
expected outliers are derived by hand below and asserted against the brute
force before anything is written.

Predicates:
  fp32_le  dx = fl32(p-q) per dim, d2 summed left to right in float32 with a
           rounding after every multiply and add, neighbour iff
           d2 <= fl32(fl32(R)^2)
  f64_lt   RTOD's own double test: |dx| < R in 1-d, sum of dx^2 < R*R otherwise

Double storage (files dbl_*.npz): points kept as float64, as RTOD keeps
them (double3 read with %lf, src/ods/optixScan.cpp:95-147), compared with
f64_lt on the doubles themselves.

Run:  python tests/golden/make_golden.py   (writes tests/golden/*.npz)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from rtod_b200 import datagen  # noqa: E402  (input generation only)

PRED = {"fp32_le": 0, "f64_lt": 1}


def window_counts(X: np.ndarray, R: float, pred: str) -> np.ndarray:
    """Uncapped neighbour counts (self included) of every point of X within X."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    d = X.shape[1]
    if pred == "fp32_le":
        Rf = np.float32(R)
        R2f = np.float32(Rf * Rf)
        s = None
        for i in range(d):
            dx = X[:, None, i] - X[None, :, i]  # float32 - float32 -> float32
            t = dx * dx
            s = t if s is None else (s + t)
        return (s <= R2f).sum(axis=1)
    X64 = X.astype(np.float64)
    if d == 1:
        return (np.abs(X64[:, None, 0] - X64[None, :, 0]) < R).sum(axis=1)
    s = None
    for i in range(d):
        dx = X64[:, None, i] - X64[None, :, i]
        t = dx * dx
        s = t if s is None else (s + t)
    return (s < R * R).sum(axis=1)


def window_counts_f64(X: np.ndarray, R: float) -> np.ndarray:
    """f64_lt counts on double coordinates (no rounding to float32)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    if X.shape[1] == 1:
        return (np.abs(X[:, None, 0] - X[None, :, 0]) < R).sum(axis=1)
    s = None
    for i in range(X.shape[1]):
        dx = X[:, None, i] - X[None, :, i]
        t = dx * dx
        s = t if s is None else (s + t)
    return (s < R * R).sum(axis=1)


def detect(points: np.ndarray, W: int, S: int, R: float, K: int, pred: str, counts=None):
    counts = counts or (lambda X: window_counts(X, R, pred))
    n = points.shape[0]
    slides = max(0, (n - W) // S) if n >= W else 0
    offsets, ids, undet = [0], [], []
    for j in range(slides):
        lo = (j + 1) * S
        c = counts(points[lo:lo + W])
        out = lo + np.nonzero(c <= K)[0]
        ids.extend(out.tolist())
        offsets.append(len(ids))
    return np.asarray(offsets, np.int64), np.asarray(ids, np.int64)


def save(name: str, points: np.ndarray, W: int, S: int, R: float, K: int, pred: str,
         expected=None, note: str = ""):
    points = np.ascontiguousarray(points, dtype=np.float32)
    if points.ndim == 1:
        points = points[:, None]
    off, ids = detect(points, W, S, R, K, pred)
    if expected is not None:
        got = [ids[off[j]:off[j + 1]].tolist() for j in range(len(off) - 1)]
        assert got == expected, f"{name}: brute force {got} != hand-derived {expected}"
    meta = dict(name=name, W=W, S=S, R=R, K=K, pred=pred, pred_id=PRED[pred], note=note,
                hand_derived=expected is not None)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), points=points, offsets=off, ids=ids,
                        meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8))
    return off, ids


def save_f64(name: str, points: np.ndarray, W: int, S: int, R: float, K: int, expected=None,
             note: str = ""):
    """A double-storage fixture (f64_lt on float64 points)."""
    points = np.ascontiguousarray(points, dtype=np.float64)
    if points.ndim == 1:
        points = points[:, None]
    off, ids = detect(points, W, S, R, K, "f64_lt", counts=lambda X: window_counts_f64(X, R))
    if expected is not None:
        got = [ids[off[j]:off[j + 1]].tolist() for j in range(len(off) - 1)]
        assert got == expected, f"{name}: brute force {got} != hand-derived {expected}"
    meta = dict(name=name, W=W, S=S, R=R, K=K, pred="f64_lt", pred_id=1, coord="f64", note=note,
                hand_derived=expected is not None)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), points=points, offsets=off, ids=ids,
                        meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8))
    return off, ids


def double_storage():
    # KAT: a pair 1e-12 inside R = 0.1 in double. As doubles they are
    # neighbours (|dx| < R); rounded to float32, 0.1 - 1e-12 becomes
    # fl32(0.1) > 0.1 and the pair is not. W = 2, S = 2, K = 1: the window
    # {2, 3} holds the pair -> no outliers with double storage.
    pts = np.array([50.0, 70.0, 0.0, 0.1 - 1e-12], np.float64)
    f32 = window_counts(pts[2:, None].astype(np.float32), 0.1, "f64_lt")
    assert f32.tolist() == [1, 1], "the pair must split when stored as float32"
    save_f64("dbl_kat_pair_inside_R", pts, 2, 2, 0.1, 1, expected=[[]],
             note="1e-12 inside R: neighbours only when stored as double")
    # KAT, 3-d: d^2 = 3 * 0.1^2 - tiny < R^2 = 0.03 + 1e-15 in double only.
    R = float(np.sqrt(0.03 + 1e-15))
    a = np.array([1.0, 2.0, 3.0])
    b = a + 0.1
    pre = np.array([[40.0, 40.0, 40.0], [60.0, 60.0, 60.0]])
    pts = np.concatenate([pre, np.stack([a, b])])
    save_f64("dbl_kat_3d", pts, 2, 2, R, 1, note="3-d pair near R in double")
    # Seeded streams whose values are not float32-representable.
    rw = datagen.random_walk(3000, 0.1, seed=21, jump_frac=0.01).astype(np.float64)
    rw = rw + np.random.default_rng(21).uniform(-1e-9, 1e-9, rw.shape)
    save_f64("dbl_walk1d", rw, 1000, 100, 0.15, 8)
    s3 = datagen.sensor_3d(2500, seed=23).astype(np.float64)
    s3 = s3 + np.random.default_rng(23).uniform(-1e-9, 1e-9, s3.shape)
    save_f64("dbl_sensor3d", s3, 1000, 250, 1.9, 12)


def known_answers():
    f = np.float32
    # KAT 1: a pair at distance exactly R = 0.5 (exact in float32, R2f = 0.25).
    # fp32_le counts it (0.25 <= 0.25); f64_lt does not (0.5 < 0.5 is false).
    # W = 2, S = 1: windows {1,2}, {2,3}.
    pts = np.array([9.0, 0.0, 0.5, 5.0], f)
    save("kat_exact_R_fp32", pts, 2, 1, 0.5, 1, "fp32_le", expected=[[], [2, 3]],
         note="pair at exactly R is a neighbour under d2 <= R2")
    save("kat_exact_R_f64", pts, 2, 1, 0.5, 1, "f64_lt", expected=[[1, 2], [2, 3]],
         note="pair at exactly R is not a neighbour under RTOD's strict <")
    # KAT 2: one ulp beyond / inside R.
    up = np.nextafter(f(0.5), f(1.0))
    dn = np.nextafter(f(0.5), f(0.0))
    pts = np.array([0.0, up, 10.0, 10.0 + dn], f)
    # windows of W=4 needs a slide: prepend 4 far points (S=4) -> window = the 4 points.
    pre = np.array([100.0, 200.0, 300.0, 400.0], f)
    save("kat_ulp_fp32", np.concatenate([pre, pts]), 4, 4, 0.5, 1, "fp32_le", expected=[[4, 5]],
         note="R+1ulp apart: outliers; R-1ulp apart: neighbours")
    # KAT 3: exactly K vs K+1 neighbours (self included). K = 3.
    # cluster A: 3 equal points (count 3 <= K -> outliers); cluster B: 4 points (count 4 -> inliers)
    body = np.array([1.0, 1.0, 1.0, 7.0, 7.0, 7.0, 7.0, 20.0], f)
    pre = np.full(8, 1000.0, f) + np.arange(8, dtype=f) * 10
    save("kat_k_boundary", np.concatenate([pre, body]), 8, 8, 0.25, 3, "fp32_le",
         expected=[[8, 9, 10, 15]], note="K points in a cluster are outliers, K+1 are not")
    # KAT 4: all outliers: points 1.0 apart, R = 0.5 -> every count is 1 <= K=1... and W = S.
    pts = np.arange(12, dtype=f)
    save("kat_all_outliers_WeqS", pts, 4, 4, 0.5, 1, "f64_lt",
         expected=[[4, 5, 6, 7], [8, 9, 10, 11]], note="W == S, every point isolated")
    # KAT 5: no outliers: all points equal (every cell dense -> nothing undetermined).
    pts = np.full(60, 3.25, f)
    save("kat_no_outliers", pts, 20, 10, 0.1, 5, "fp32_le", expected=[[], [], [], []],
         note="all points identical: empty outlier and undetermined sets")
    # KAT 6: 3-d exact distances with power-of-two coordinates, R = 0.5, K = 1.
    #  a=(0,0,0) b=(0.5,0,0): d2 = 0.25 -> neighbours (fp32_le), not (f64_lt)
    #  c=(10,10,10) e=(10.25,10.25,10.25): d2 = 0.1875 -> neighbours in both
    #  g=(20,20,20) h=(20.5,20.25,20): d2 = 0.3125 -> not neighbours
    body = np.array([[0, 0, 0], [0.5, 0, 0], [10, 10, 10], [10.25, 10.25, 10.25],
                     [20, 20, 20], [20.5, 20.25, 20]], f)
    pre = np.full((6, 3), -50.0, f) + np.arange(6, dtype=f)[:, None] * 7
    pts = np.concatenate([pre, body])
    save("kat_3d_fp32", pts, 6, 6, 0.5, 1, "fp32_le", expected=[[10, 11]])
    save("kat_3d_f64", pts, 6, 6, 0.5, 1, "f64_lt", expected=[[6, 7, 10, 11]])
    # KAT 7: 8-d, the neighbour pair differs by 0.25 in four dims (d2 = 0.25).
    a = np.zeros(8, f)
    b = np.array([0.25, 0.25, 0.25, 0.25, 0, 0, 0, 0], f)
    c = np.array([0.25, 0.25, 0.25, 0.25, 0.25, 0, 0, 0], f) + 5
    e = np.full(8, 5.0, f)
    pre = np.full((4, 8), -40.0, f) + np.arange(4, dtype=f)[:, None] * 9
    save("kat_8d_fp32", np.concatenate([pre, np.stack([a, b, c, e])]), 4, 4, 0.5, 1, "fp32_le",
         expected=[[6, 7]], note="8-d: d2 = 0.25 neighbour, d2 = 0.3125 not")
    # KAT 8: K >= W -> every point is an outlier.
    pts = np.zeros(10, f)
    save("kat_K_ge_W", pts, 5, 5, 1.0, 5, "fp32_le", expected=[[5, 6, 7, 8, 9]])


def seeded_streams():
    rw = datagen.random_walk(3000, 0.1, seed=11, jump_frac=0.01)
    save("walk1d_fp32", rw, 1000, 100, 0.15, 8, "fp32_le")
    save("walk1d_f64", rw, 1000, 100, 0.15, 8, "f64_lt")
    gm = datagen.gaussian_mixture(2400, seed=12)
    save("gmm1d_fp32", gm, 800, 200, 0.004, 6, "fp32_le")
    s3 = datagen.sensor_3d(2500, seed=13)
    save("sensor3d_fp32", s3, 1000, 250, 1.9, 12, "fp32_le")
    save("sensor3d_f64", s3, 1000, 250, 1.9, 12, "f64_lt")
    w8 = datagen.random_walk(1800, 0.1, seed=14, dim=8)
    save("walk8d_fp32", w8, 600, 200, 0.55, 5, "fp32_le")
    w3 = datagen.random_walk(2000, 0.1, seed=15, dim=3)
    save("walk3d_fp32_K0", w3, 500, 500, 0.3, 0, "fp32_le")
    # Quantised values: many exact ties and many pairs at exactly R.
    q = (np.round(datagen.random_walk(2000, 0.3, seed=16) * 4) / 4).astype(np.float32)
    save("quantised1d_fp32", q, 400, 100, 0.5, 4, "fp32_le")
    save("quantised1d_f64", q, 400, 100, 0.5, 4, "f64_lt")


if __name__ == "__main__":
    known_answers()
    seeded_streams()
    double_storage()
    for fn in sorted(os.listdir(HERE)):
        if fn.endswith(".npz"):
            z = np.load(os.path.join(HERE, fn))
            print(f"{fn:32s} n={z['points'].shape} slides={len(z['offsets']) - 1} "
                  f"outliers={len(z['ids'])}")
