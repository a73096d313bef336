"""Python front end of the detector: the run surface of RTOD's optixScan.

``Detector`` mirrors the parameters of ``optixScan`` (``--window --slide
--R --K``, src/ods/optixScan.cpp:149-212) and its compile-time switches
(``DIMENSION``, ``OPTIMIZATION``, src/ods/optixScan.h:10-24) and reproduces
its slide loop (``detect_outlier``, src/ods/optixScan.cpp:1019-1126): the
first W points fill the window, every later slide of S points yields the
outliers of the new window. Results are sorted global stream indices
(``Detector.ring_slots`` converts them to RTOD's ring-slot IDs). All work
runs in librtod.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native
from ._native import Config, Times, check, lib


def _as_points(points, dim: int, f64: bool = False):
    """(pointer, n, keepalive) for a point-major float32 (float64 with f64)
    array: a numpy array (host) or a CUDA tensor exposing data_ptr() (device)."""
    if hasattr(points, "data_ptr") and hasattr(points, "is_cuda"):
        t = points
        want = "torch.float64" if f64 else "torch.float32"
        if t.dtype.__repr__() != want or not t.is_contiguous():
            raise TypeError(f"device points must be a contiguous {want[6:]} tensor")
        n = t.numel() // dim
        if n * dim != t.numel():
            raise ValueError(f"tensor size {t.numel()} is not a multiple of dim={dim}")
        return ctypes.c_void_p(t.data_ptr()), n, t
    a = np.ascontiguousarray(points, dtype=np.float64 if f64 else np.float32)
    if a.ndim == 1 and dim == 1:
        a = a[:, None]
    if a.ndim != 2 or a.shape[1] != dim:
        raise ValueError(f"expected points of shape (n, {dim}), got {a.shape}")
    return a.ctypes.data_as(ctypes.c_void_p), a.shape[0], a


@dataclass
class RunResult:
    """Outliers of every slide of a stream, in CSR form."""
    offsets: np.ndarray  # int64 [slides + 1]
    ids: np.ndarray      # int64 [offsets[-1]]
    times: dict = field(default_factory=dict)

    @property
    def slides(self) -> int:
        return len(self.offsets) - 1

    def slide(self, j: int) -> np.ndarray:
        return self.ids[self.offsets[j]:self.offsets[j + 1]]


# Kernels of the span engine timed in each stage slot of rtod_profile_run.
SPAN_STAGES = {"k_hist": "k_span_hist", "k_scan": "k_span_scan+k_span_prefix",
               "k_scatter": "k_span_scatter", "k_count": "k_span_classify", "k_compact": "k_span_count",
               "k_train": "k_span_compact"}


class Detector:
    """Sliding-window distance outlier detector on one CUDA device.

    A point of the window is an outlier when at most K window points (itself
    included) lie within distance R of it.
    """

    def __init__(self, window: int, slide: int, R: float, K: int, dim: int = 1, opt: int = 2,
                 pred: str = "fp32_le", router: bool = False, tuner: bool = False,
                 cells_per_r: int = 0, block_warps: int = 0, use_graph: bool = True,
                 batch: int = 0, device: int = 0, engine: str = "auto", coord: str = "f32",
                 count: str = "auto", pipeline: str = "staged"):
        cfg = Config()
        check(lib().rtod_config_init(ctypes.byref(cfg)))
        cfg.window, cfg.slide, cfg.R, cfg.K, cfg.dim, cfg.opt = window, slide, R, K, dim, opt
        cfg.pred = _native.PRED[pred]
        cfg.router, cfg.tuner = int(router), int(tuner)
        cfg.cells_per_r, cfg.block_warps = cells_per_r, block_warps
        cfg.use_graph, cfg.device, cfg.batch = int(use_graph), device, batch
        cfg.engine = _native.ENGINE[engine]
        cfg.coord = _native.COORD[coord]
        cfg.count = _native.COUNT[count]
        cfg.pipeline = _native.PIPELINE[pipeline]
        self.f64 = coord == "f64"
        self.cfg = cfg
        self.window, self.slide, self.R, self.K, self.dim = window, slide, R, K, dim
        self._h = ctypes.c_void_p()
        check(lib().rtod_create(ctypes.byref(cfg), ctypes.byref(self._h)))

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if self._h:
            lib().rtod_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- streaming --------------------------------------------------------
    def push(self, points) -> None:
        """Appends W points (first call) or S points (each later call)."""
        ptr, n, keep = _as_points(points, self.dim, self.f64)
        push = lib().rtod_push_slide_f64 if self.f64 else lib().rtod_push_slide
        check(push(self._h, ptr, n))
        del keep

    def detect(self, times: bool = False):
        """Outliers (sorted global indices) of the window after the last push."""
        out = self.__dict__.get("_detect_out")
        if out is None:  # one buffer per detector: a window has at most W outliers
            out = self._detect_out = np.empty(self.window, np.int64)
        n_out = ctypes.c_int64()
        t = Times()
        check(lib().rtod_detect(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size,
                                ctypes.byref(n_out), ctypes.byref(t) if times else None))
        ids = out[:n_out.value].copy()
        return (ids, t.as_dict()) if times else ids

    def run(self, points, max_slides: int = 10000, times: bool = False, ids_cap: int | None = None,
            out_ids=None) -> RunResult:
        """Processes a whole stream (host array or CUDA tensor) like RTOD's
        detect_outlier: fill with the first W points, then detect up to
        max_slides slides (RTOD caps the loop at 10000, optixScan.cpp:1045)."""
        ptr, n, keep = _as_points(points, self.dim, self.f64)
        slides = max(0, (n - self.window) // self.slide) if n >= self.window else 0
        if max_slides is not None and max_slides >= 0:
            slides = min(slides, max_slides)
        off = np.zeros(slides + 1, np.int64)
        if ids_cap is None:
            ids_cap = max(1, slides * self.window)
        if out_ids is None:
            out = np.empty(ids_cap, np.int64)
            out_ptr = out.ctypes.data_as(ctypes.c_void_p)
        elif isinstance(out_ids, np.ndarray):
            if out_ids.dtype != np.int64 or not out_ids.flags.c_contiguous:
                raise TypeError("out_ids must be a contiguous int64 array")
            out = out_ids
            ids_cap = min(ids_cap, out.size)
            out_ptr = out.ctypes.data_as(ctypes.c_void_p)
        else:
            out = out_ids
            ids_cap = min(ids_cap, out.numel())
            out_ptr = ctypes.c_void_p(out_ids.data_ptr())
        ns = ctypes.c_int64()
        t = Times()
        fn = lib().rtod_run_f64 if self.f64 else lib().rtod_run
        check(fn(self._h, ptr, n, -1 if max_slides is None else max_slides,
                             off.ctypes.data_as(ctypes.c_void_p), out_ptr, ids_cap,
                             ctypes.byref(ns), ctypes.byref(t) if times else None))
        del keep
        ids = out[:off[-1]] if out_ids is not None else out[:off[-1]].copy()
        return RunResult(off, ids, t.as_dict() if times else {})

    @property
    def stats(self) -> dict:
        a = (ctypes.c_int64 * 5)()
        check(lib().rtod_get_stats(self._h, a))
        return {"launches": a[0], "graph_replays": a[1], "slides": a[2], "undetermined": a[3],
                "device_bytes": a[4]}

    def profile(self, points, max_slides: int = -1) -> dict:
        """Average device ms per slide of each pipeline kernel (diagnostic run
        on a fresh handle; every kernel launched on its own with CUDA events)."""
        ptr, n, keep = _as_points(points, self.dim)
        ms = (ctypes.c_double * 8)()
        check(lib().rtod_profile_run(self._h, ptr, n, max_slides, ms, 8))
        del keep
        span = self.tuning["engine"] == "span"
        out = {}
        for i in range(8):
            name = lib().rtod_kernel_name(i)
            if name is None:
                break
            name = name.decode()
            out[SPAN_STAGES.get(name, name) if span else name] = ms[i]
        return out

    def reset(self) -> None:
        check(lib().rtod_reset(self._h))

    @property
    def stream_engine(self) -> dict:
        """Engine of push/detect ("grid": the streaming grid engine, or
        "window"), builds of the grid from the ring, its pool slots and the
        largest bin occupancy of the last counted window."""
        a = (ctypes.c_int64 * 4)()
        check(lib().rtod_get_stream_engine(self._h, a))
        return {"engine": _native.ENGINE_NAME.get(a[0], a[0]), "builds": a[1], "pool": a[2], "max_occ": a[3]}

    def set_grid_pool(self, slots: int) -> None:
        """Pool slots of the streaming grid's first build (before the first push)."""
        check(lib().rtod_set_grid_pool(self._h, int(slots)))

    def router_info(self) -> dict:
        """Learned-router state: parameters, training steps and routing counters."""
        params = np.zeros(int(lib().rtod_mlp_param_count()), np.float32)
        info = np.zeros(6, np.float64)
        check(lib().rtod_router_info(self._h, params.ctypes.data_as(ctypes.c_void_p),
                                     info.ctypes.data_as(ctypes.c_void_p)))
        return {"params": params, "steps": int(info[0]), "last_loss": float(info[1]),
                "routed_early": int(info[2]), "routed_sweep": int(info[3]),
                "misrouted": int(info[4]), "threshold": float(info[5])}

    def set_router_threshold(self, threshold: float) -> None:
        """Routing threshold of the learned router (see rtod_router_set_threshold)."""
        check(lib().rtod_router_set_threshold(self._h, float(threshold)))

    @property
    def slides_done(self) -> int:
        return int(lib().rtod_slides_done(self._h))

    @property
    def tuning(self) -> dict:
        a = (ctypes.c_int32 * 5)()
        check(lib().rtod_get_tuning(self._h, a))
        return {"cells_per_r": a[0], "block_warps": a[1], "hashed_dims": a[2], "batch": a[3],
                "engine": _native.ENGINE_NAME.get(a[4], a[4])}

    @property
    def count_mode(self) -> str:
        """Window-engine count: "point" (warp per point) or "group" (warp per bin)."""
        m = ctypes.c_int32()
        check(lib().rtod_get_count_mode(self._h, ctypes.byref(m)))
        return _native.COUNT_NAME.get(m.value, m.value)

    def ring_slots(self, ids: np.ndarray) -> np.ndarray:
        """RTOD's outlier IDs (ring slots, optixScan.cpp:1097) for global indices."""
        return np.asarray(ids, np.int64) % self.window


class BatchDetector:
    """Many independent streams advanced together, one slide per step; each
    step detects every stream that was pushed a slide, in one replay of a
    captured CUDA graph (streams grouped by dimension and predicate).

    ``streams`` is a list of dicts with the Detector parameters (window,
    slide, R, K, dim, opt, pred, count, cells_per_r, block_warps); ``router``
    switches the shared learned router on for all of them; ``tuner`` lets the
    autotuner pick each group's cell width, count block shape and (beyond 3
    dimensions) count mode over the first steps."""

    def __init__(self, streams, router: bool = False, device: int = 0, tuner: bool = False):
        n = len(streams)
        cfgs = (Config * n)()
        for i, st in enumerate(streams):
            check(lib().rtod_config_init(ctypes.byref(cfgs[i])))
            c = cfgs[i]
            c.window, c.slide, c.R, c.K = st["window"], st["slide"], st["R"], st["K"]
            c.dim, c.opt = st.get("dim", 1), st.get("opt", 2)
            c.pred = _native.PRED[st.get("pred", "fp32_le")]
            c.count = _native.COUNT[st.get("count", "auto")]
            c.pipeline = _native.PIPELINE[st.get("pipeline", "staged")]
            c.cells_per_r, c.block_warps = st.get("cells_per_r", 0), st.get("block_warps", 0)
            c.router, c.device, c.tuner = int(router), device, int(tuner)
        self.streams = [dict(s) for s in streams]
        self._b = ctypes.c_void_p()
        check(lib().rtod_batch_create(cfgs, n, ctypes.byref(self._b)))
        self._cap = sum(int(s["window"]) for s in streams)
        self._out = np.empty(self._cap, np.int64)

    def close(self) -> None:
        if self._b:
            lib().rtod_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def push(self, s: int, points) -> None:
        ptr, n, keep = _as_points(points, int(self.streams[s].get("dim", 1)))
        check(lib().rtod_batch_push(self._b, s, ptr, n))
        del keep

    @property
    def tuning(self) -> list:
        """Per group of streams: its dimension, predicate, cells per R, count
        block warps, count mode and whether the autotuner has settled it."""
        a = (ctypes.c_int32 * (6 * 64))()
        ng = lib().rtod_batch_get_tuning(self._b, a, 64)
        if ng < 0:
            check(ng)
        return [{"dim": a[6 * i], "pred": a[6 * i + 1], "cells_per_r": a[6 * i + 2], "block_warps": a[6 * i + 3],
                 "count": _native.COUNT_NAME.get(a[6 * i + 4], a[6 * i + 4]), "settled": bool(a[6 * i + 5])}
                for i in range(min(ng, 64))]

    def step(self):
        """Per-stream sorted outlier IDs of this step (empty for streams that
        sat the step out)."""
        off = np.zeros(len(self.streams) + 1, np.int64)
        n = ctypes.c_int64()
        check(lib().rtod_batch_step(self._b, off.ctypes.data_as(ctypes.c_void_p),
                                    self._out.ctypes.data_as(ctypes.c_void_p), self._cap,
                                    ctypes.byref(n)))
        return [self._out[off[i]:off[i + 1]].copy() for i in range(len(self.streams))]

    @property
    def stats(self) -> dict:
        a = (ctypes.c_int64 * 5)()
        check(lib().rtod_batch_stats(self._b, a))
        return {"steps": a[0], "launches": a[1], "detections": a[2], "groups": a[3], "pair_tests": a[4]}
