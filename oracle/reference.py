"""ctypes front end of RTOD's own host code, built by oracle/ref/Makefile into
oracle/_ref/ (TEST INFRASTRUCTURE ONLY).

The build compiles RTOD's src/ods/optixScan.cpp from an RTOD checkout; it is
only possible where that checkout exists, and its outputs are committed as
fixtures under tests/golden/ (ref_*.npz) by tests/golden/make_ref_golden.py.
Nothing on the GPU path, in bench.py or in smoke() loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REF_DEFAULT = "/root/reference"


def lib_path(dim: int) -> str:
    return os.path.join(OUT, f"librtod_ref_d{dim}.so")


def available() -> bool:
    return all(os.path.exists(lib_path(d)) for d in (1, 3))


def build(ref: str | None = None, force: bool = False) -> bool:
    """Builds both libraries when the RTOD sources are present; returns
    whether they are available afterwards."""
    ref = ref or os.environ.get("RTOD_REF", REF_DEFAULT)
    src = os.path.join(ref, "src", "ods", "optixScan.cpp")
    if not os.path.exists(src):
        return available()
    args = ["make", "-s", "-C", os.path.join(HERE, "ref"), f"REF={ref}"]
    if force:
        args.append("-B")
    subprocess.run(args, check=True)
    return available()


_libs: dict[int, ctypes.CDLL] = {}


def _lib(dim: int) -> ctypes.CDLL:
    if dim not in _libs:
        L = ctypes.CDLL(lib_path(dim))
        vp, i64, i32, f64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double
        L.rtod_ref_detect.restype = i64
        L.rtod_ref_detect.argtypes = [vp, i64, i32, i32, f64, i32, i32, vp, vp, i64, vp, vp, i64, vp,
                                      ctypes.c_char_p]
        _libs[dim] = L
    return _libs[dim]


def detect(points: np.ndarray, W: int, S: int, R: float, K: int, brute: bool = True):
    """Runs RTOD's detect_outlier (and, with brute, its check_outlier on every
    slide) over a 1-d or 3-d stream of doubles. Returns
    (offsets, ids, b_offsets, b_ids, stats): CSR per-slide sorted global
    indices of RTOD's picked outliers and of check_outlier's outliers;
    stats = [undetermined points summed over slides, margin events, slides]."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    if pts.ndim == 1:
        pts = pts[:, None]
    n, d = pts.shape
    if d not in (1, 3):
        raise ValueError("RTOD supports 1-d and 3-d points")
    slides = (n - W) // S
    cap = max(1, slides * W)
    off = np.zeros(slides + 1, np.int64)
    ids = np.zeros(cap, np.int64)
    boff = np.zeros(slides + 1, np.int64)
    bids = np.zeros(cap if brute else 1, np.int64)
    stats = np.zeros(3, np.int64)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    with tempfile.TemporaryDirectory() as tmp:
        r = _lib(d).rtod_ref_detect(p(pts), n, W, S, float(R), K, 1 if brute else 0, p(off), p(ids), cap,
                                    p(boff), p(bids), bids.size, p(stats), tmp.encode())
    if r < 0:
        raise RuntimeError(f"rtod_ref_detect failed with code {r}")
    if r != slides:
        raise RuntimeError(f"RTOD ran {r} slides, expected {slides}")
    out = (off, ids[:off[-1]].copy())
    bout = (boff, bids[:boff[-1]].copy()) if brute else (None, None)
    return out[0], out[1], bout[0], bout[1], stats
