"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference
legs import this module. The product package (rtod_b200) never does.
Pinned to RTOD's own code (tests/golden/ref_*.npz): see the header of
rtod_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "librtod_oracle.so")

PRED = {"fp32_le": 0, "f64_lt": 1}
ENGINE = {"brute": 0, "grid": 1, "grid_nofilter": 2}

_lib = None


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("rtod_oracle.cpp", "mlp_oracle.cpp", "Makefile")]
    if force or not os.path.exists(LIB_PATH) or any(
            os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        i64, i32, f64, vp = ctypes.c_int64, ctypes.c_int32, ctypes.c_double, ctypes.c_void_p
        L.oracle_detect.restype = i64
        L.oracle_detect.argtypes = [vp, i64, i32, i64, i64, f64, i32, i32, i32, i32, i64, vp, vp, i64, vp]
        L.oracle_window_counts.restype = i32
        L.oracle_window_counts.argtypes = [vp, i64, i32, i64, i64, f64, i32, vp]
        L.oracle_detect_f64.restype = i64
        L.oracle_detect_f64.argtypes = [vp, i64, i32, i64, i64, f64, i32, i32, i32, i32, i64, vp, vp, i64, vp]
        L.oracle_pred.restype = i32
        L.oracle_pred.argtypes = [vp, vp, i32, f64, i32]
        L.oracle_pred_f64.restype = i32
        L.oracle_pred_f64.argtypes = [vp, vp, i32, f64]
        L.oracle_mlp_param_count.restype = i32
        L.oracle_mlp_param_count.argtypes = [i32]
        L.oracle_mlp_forward.restype = i32
        L.oracle_mlp_forward.argtypes = [vp, i32, vp, i64, vp]
        L.oracle_mlp_loss_grad.restype = i32
        L.oracle_mlp_loss_grad.argtypes = [vp, i32, vp, vp, i64, vp, vp]
        L.oracle_mlp_adam.restype = i32
        L.oracle_mlp_adam.argtypes = [vp, vp, vp, vp, i32, i32, f64, f64, f64, f64]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def detect(points: np.ndarray, W: int, S: int, R: float, K: int, pred="fp32_le", engine="grid",
           threads: int = 1, max_slides: int = 10000, ids_cap: int | None = None, f64: bool = False):
    """Per-slide sorted outlier indices in CSR form: (offsets, ids, stats).
    stats = [undetermined points summed over slides, pair tests, slides].
    f64: the points are kept as double (RTOD's storage) and compared with
    RTOD's double predicate (pred must be "f64_lt")."""
    pts = np.ascontiguousarray(points, dtype=np.float64 if f64 else np.float32)
    if pts.ndim == 1:
        pts = pts[:, None]
    n, d = pts.shape
    slides = max(0, (n - W) // S) if n >= W else 0
    if max_slides >= 0:
        slides = min(slides, max_slides)
    if ids_cap is None:
        ids_cap = max(1, slides * W)
    off = np.zeros(slides + 1, np.int64)
    ids = np.zeros(ids_cap, np.int64)
    stats = np.zeros(3, np.int64)
    fn = lib().oracle_detect_f64 if f64 else lib().oracle_detect
    r = fn(_ptr(pts), n, d, W, S, float(R), K,
                            PRED[pred] if isinstance(pred, str) else int(pred),
                            ENGINE[engine], threads, max_slides, _ptr(off), _ptr(ids), ids_cap,
                            _ptr(stats))
    if r < 0:
        raise ValueError(f"oracle_detect failed with code {r}")
    return off, ids[:off[-1]].copy(), stats


def window_counts(points: np.ndarray, lo: int, W: int, R: float, pred="fp32_le") -> np.ndarray:
    pts = np.ascontiguousarray(points, dtype=np.float32)
    if pts.ndim == 1:
        pts = pts[:, None]
    out = np.zeros(W, np.int32)
    r = lib().oracle_window_counts(_ptr(pts), pts.shape[0], pts.shape[1], lo, W, float(R),
                                   PRED[pred], _ptr(out))
    if r != 0:
        raise ValueError("oracle_window_counts failed")
    return out


def pred(p, q, R: float, mode="fp32_le") -> bool:
    p = np.ascontiguousarray(p, dtype=np.float32).ravel()
    q = np.ascontiguousarray(q, dtype=np.float32).ravel()
    return bool(lib().oracle_pred(_ptr(p), _ptr(q), p.size, float(R), PRED[mode]))


def pred_f64(p, q, R: float) -> bool:
    """RTOD's double predicate on double coordinates."""
    p = np.ascontiguousarray(p, dtype=np.float64).ravel()
    q = np.ascontiguousarray(q, dtype=np.float64).ravel()
    return bool(lib().oracle_pred_f64(_ptr(p), _ptr(q), p.size, float(R)))


def mlp_param_count(B: int = 4) -> int:
    return int(lib().oracle_mlp_param_count(B))


def mlp_forward(params: np.ndarray, X: np.ndarray, B: int = 4) -> np.ndarray:
    params = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    out = np.zeros((X.shape[0], B), np.float64)
    if lib().oracle_mlp_forward(_ptr(params), B, _ptr(X), X.shape[0], _ptr(out)) != 0:
        raise ValueError("oracle_mlp_forward failed")
    return out


def mlp_loss_grad(params: np.ndarray, X: np.ndarray, y: np.ndarray, B: int = 4):
    params = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    grad = np.zeros(params.size, np.float64)
    loss = np.zeros(1, np.float64)
    if lib().oracle_mlp_loss_grad(_ptr(params), B, _ptr(X), _ptr(y), X.shape[0], _ptr(loss),
                                  _ptr(grad)) != 0:
        raise ValueError("oracle_mlp_loss_grad failed")
    return float(loss[0]), grad


def mlp_adam(params, m, v, grad, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    p = np.array(params, np.float32)
    m = np.array(m, np.float32)
    v = np.array(v, np.float32)
    g = np.ascontiguousarray(grad, np.float32)
    lib().oracle_mlp_adam(_ptr(p), _ptr(m), _ptr(v), _ptr(g), p.size, t, lr, b1, b2, eps)
    return p, m, v
