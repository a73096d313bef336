"""Seeded synthetic streams standing in for RTOD's missing datasets.

RTOD's experiments read three text files that are not in its repository
(``.MISSING_LARGE_BLOBS:1-3``): ``stock.txt`` (STK, 1-d), ``tao.txt`` (TAO,
3-d) and ``gaussian.txt`` (GAU, 1-d). The generators below produce streams
with the same lengths and run parameters as ``script/run.py:13,25,37`` and
the value distributions described for each workload. Values are drawn in
float64 with numpy's PCG64 and cast to float32 once; points are returned
point-major as an ``(n, d)`` float32 array, the layout of RTOD's ``double3
vertices[]`` (``src/ods/optixScan.cpp:95-147``) at single precision.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass(frozen=True)
class Workload:
    """One stream plus the detector parameters it is run with."""

    name: str
    points: np.ndarray  # (n, d) float32
    window: int
    slide: int
    R: float
    K: int

    @property
    def dim(self) -> int:
        return int(self.points.shape[1])

    @property
    def n(self) -> int:
        return int(self.points.shape[0])

    @property
    def slides(self) -> int:
        return max(0, (self.n - self.window) // self.slide)


def random_walk(n: int, step_sigma: float, seed: int, jump_frac: float = 0.0,
                jump_half_width: float = 5.0, dim: int = 1) -> np.ndarray:
    """x_0 = 0, x_t = x_{t-1} + N(0, step_sigma) per dimension; a fraction
    ``jump_frac`` of the steps also gets a U(-w, w) level jump."""
    rng = np.random.Generator(np.random.PCG64(seed))
    steps = rng.normal(0.0, step_sigma, size=(n, dim))
    if jump_frac > 0:
        hit = rng.random(n) < jump_frac
        steps[hit] += rng.uniform(-jump_half_width, jump_half_width, size=(int(hit.sum()), dim))
    steps[0] = 0.0
    return np.cumsum(steps, axis=0).astype(np.float32)


def gaussian_mixture(n: int, seed: int, means=(0.0, 0.3, 0.7), sigma: float = 0.02,
                     weights=(0.5, 0.3, 0.2), noise_frac: float = 0.01,
                     noise_lo: float = -1.0, noise_hi: float = 2.0, dim: int = 1) -> np.ndarray:
    """i.i.d. draws from a 1-d Gaussian mixture (per dimension), with a fraction
    of the points replaced by U(noise_lo, noise_hi)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    comp = rng.choice(len(means), size=n, p=np.asarray(weights) / np.sum(weights))
    x = np.asarray(means)[comp][:, None] + rng.normal(0.0, sigma, size=(n, dim))
    hit = rng.random(n) < noise_frac
    x[hit] = rng.uniform(noise_lo, noise_hi, size=(int(hit.sum()), dim))
    return x.astype(np.float32)


def sensor_3d(n: int, seed: int, period: float = 1440.0, amp: float = 10.0,
              noise_frac: float = 0.01, noise_half_width: float = 30.0) -> np.ndarray:
    """Each dimension d is amp*sin(2*pi*t/period + phi_d) + N(0, 1), with
    phi_d = 2*pi*d/3; a fraction of points is replaced by U(-w, w)^3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.arange(n, dtype=np.float64)[:, None]
    phi = 2.0 * math.pi * np.arange(3, dtype=np.float64)[None, :] / 3.0
    x = amp * np.sin(2.0 * math.pi * t / period + phi) + rng.normal(0.0, 1.0, size=(n, 3))
    hit = rng.random(n) < noise_frac
    x[hit] = rng.uniform(-noise_half_width, noise_half_width, size=(int(hit.sum()), 3))
    return x.astype(np.float32)


def small_walk() -> Workload:
    """1-d random walk, 200,000 values, W=10,000, S=500, R=0.45, K=50."""
    return Workload("walk-1d-W10k", random_walk(200_000, 0.1, seed=0), 10_000, 500, 0.45, 50)


def stock_like() -> Workload:
    """STK stand-in: 1-d random walk with 0.5% U(-5,5) jumps, 1,048,572 values,
    W=100,000, S=5,000, R=0.45, K=50 (script/run.py:25)."""
    return Workload("stk-1d-W100k", random_walk(1_048_572, 0.1, seed=1, jump_frac=0.005),
                    100_000, 5_000, 0.45, 50)


def sensor_like() -> Workload:
    """TAO stand-in: 3-d, 575,468 points, W=10,000, S=500, R=1.9, K=50 (script/run.py:37)."""
    return Workload("tao-3d-W10k", sensor_3d(575_468, seed=2), 10_000, 500, 1.9, 50)


def gaussian_like(K: int = 50) -> Workload:
    """GAU stand-in: 1-d Gaussian mixture, 1,000,000 values, W=100,000, S=5,000,
    R=0.028 (script/run.py:13); K swept over {30, 50, 70}."""
    return Workload(f"gau-1d-W100k-K{K}", gaussian_mixture(1_000_000, seed=3), 100_000, 5_000,
                    0.028, K)


def radius_for_outlier_fraction(window: np.ndarray, K: int, frac: float, seed: int,
                                sample: int = 4096) -> float:
    """R such that about ``frac`` of the window's points have at most K
    neighbours (self included) within R: the (1-frac) quantile of the distance
    to the (K+1)-th nearest neighbour, estimated on a sample of query points."""
    from scipy.spatial import cKDTree  # generator-time dependency only

    rng = np.random.Generator(np.random.PCG64(seed))
    q = window[rng.choice(len(window), size=min(sample, len(window)), replace=False)]
    dist, _ = cKDTree(window.astype(np.float64)).query(q.astype(np.float64), k=K + 1)
    return float(np.quantile(dist[:, -1], 1.0 - frac)) * 1.0001


def batched_streams(count: int = 64, slides: int = 40, seed0: int = 4, K: int = 50,
                    outlier_frac: float = 0.02, w_lo: int = 5_000, w_hi: int = 200_000):
    """Many independent streams of uneven shape: W log-uniform in [w_lo, w_hi]
    rounded to a multiple of 20, S = W/20, d in {1, 3, 8}, random-walk or
    Gaussian-mixture values, R chosen so that about 2% of the first window's
    points are outliers, K = 50. Each stream holds W + slides*S points."""
    out = []
    for i in range(count):
        rng = np.random.Generator(np.random.PCG64(seed0 + i))
        W = int(round(math.exp(rng.uniform(math.log(w_lo), math.log(w_hi))) / 20.0)) * 20
        S = W // 20
        d = int(rng.choice([1, 3, 8]))
        n = W + slides * S
        if rng.random() < 0.5:
            pts = random_walk(n, 0.1, seed=seed0 + 1000 + i, dim=d)
            kind = "walk"
        else:
            pts = gaussian_mixture(n, seed=seed0 + 1000 + i, dim=d)
            kind = "gmm"
        R = radius_for_outlier_fraction(pts[:W], K, outlier_frac, seed=seed0 + 2000 + i)
        out.append(Workload(f"batch{i}-{kind}-d{d}-W{W}", pts, W, S, R, K))
    return out
