"""ctypes binding of librtod.so (the C ABI declared in include/rtod.h).

The library is loaded from this package folder. There is no fallback: if the
shared object is missing or cannot be loaded, importing the detector fails
with an error that says how to build it.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "librtod.so")

RTOD_OK = 0
ERRORS = {
    -1: "RTOD_ERR_CONFIG", -2: "RTOD_ERR_ARG", -3: "RTOD_ERR_CUDA", -4: "RTOD_ERR_CAPACITY",
    -5: "RTOD_ERR_INPUT", -6: "RTOD_ERR_STATE", -7: "RTOD_ERR_TIMEOUT", -8: "RTOD_ERR_NODEV",
}
PRED = {"fp32_le": 0, "f64_lt": 1}


class RtodError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


ENGINE = {"auto": 0, "window": 1, "span": 2, "grid": 3}
COORD = {"f32": 0, "f64": 1}
COUNT = {"auto": 0, "point": 1, "group": 2}
COUNT_NAME = {1: "point", 2: "group"}
PIPELINE = {"staged": 0, "fused": 1}
ENGINE_NAME = {1: "window", 2: "span", 3: "grid"}


class Config(ctypes.Structure):
    _fields_ = [
        ("window", ctypes.c_int64), ("slide", ctypes.c_int64), ("R", ctypes.c_double),
        ("K", ctypes.c_int32), ("dim", ctypes.c_int32), ("opt", ctypes.c_int32),
        ("pred", ctypes.c_int32), ("router", ctypes.c_int32), ("tuner", ctypes.c_int32),
        ("cells_per_r", ctypes.c_int32), ("block_warps", ctypes.c_int32),
        ("use_graph", ctypes.c_int32), ("device", ctypes.c_int32), ("batch", ctypes.c_int32),
        ("engine", ctypes.c_int32), ("coord", ctypes.c_int32), ("count", ctypes.c_int32),
        ("pipeline", ctypes.c_int32),
    ]


class Times(ctypes.Structure):
    _fields_ = [
        ("copy_new_points_h2d", ctypes.c_double), ("copy_filtered_points_h2d", ctypes.c_double),
        ("copy_outlier_d2h", ctypes.c_double), ("prepare_cell", ctypes.c_double),
        ("build_bvh", ctypes.c_double), ("detect_outlier", ctypes.c_double),
        ("total", ctypes.c_double), ("undetermined_per_slide", ctypes.c_double),
        ("slides", ctypes.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None

# (name, restype, argtypes) of every exported entry point of include/rtod.h
_vp, _i64, _i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
SIGNATURES = [
    ("rtod_config_init", _i32, [ctypes.POINTER(Config)]),
    ("rtod_create", _i32, [ctypes.POINTER(Config), ctypes.POINTER(_vp)]),
    ("rtod_push_slide", _i32, [_vp, _vp, _i64]),
    ("rtod_push_slide_f64", _i32, [_vp, _vp, _i64]),
    ("rtod_detect", _i32, [_vp, _vp, _i64, ctypes.POINTER(_i64), ctypes.POINTER(Times)]),
    ("rtod_run", _i32, [_vp, _vp, _i64, _i64, _vp, _vp, _i64, ctypes.POINTER(_i64),
                        ctypes.POINTER(Times)]),
    ("rtod_run_f64", _i32, [_vp, _vp, _i64, _i64, _vp, _vp, _i64, ctypes.POINTER(_i64),
                            ctypes.POINTER(Times)]),
    ("rtod_reset", _i32, [_vp]),
    ("rtod_slides_done", _i64, [_vp]),
    ("rtod_get_tuning", _i32, [_vp, _vp]),
    ("rtod_get_count_mode", _i32, [_vp, ctypes.POINTER(_i32)]),
    ("rtod_check_bounded_wait", _i32, [_i32, ctypes.POINTER(_i32), ctypes.POINTER(ctypes.c_double)]),
    ("rtod_get_stats", _i32, [_vp, _vp]),
    ("rtod_get_stream_engine", _i32, [_vp, _vp]),
    ("rtod_set_grid_pool", _i32, [_vp, _i64]),
    ("rtod_profile_run", _i32, [_vp, _vp, _i64, _i64, _vp, _i32]),
    ("rtod_kernel_name", ctypes.c_char_p, [_i32]),
    ("rtod_router_info", _i32, [_vp, _vp, _vp]),
    ("rtod_router_set_threshold", _i32, [_vp, ctypes.c_float]),
    ("rtod_detect_window_static", _i32, [_vp, _i64, _i32, ctypes.c_double, _i32, _i32, _vp,
                                         ctypes.POINTER(_i64), _vp]),
    ("rtod_batch_create", _i32, [_vp, _i32, ctypes.POINTER(_vp)]),
    ("rtod_batch_push", _i32, [_vp, _i32, _vp, _i64]),
    ("rtod_batch_step", _i32, [_vp, _vp, _vp, _i64, ctypes.POINTER(_i64)]),
    ("rtod_batch_stats", _i32, [_vp, _vp]),
    ("rtod_batch_get_tuning", _i32, [_vp, _vp, _i32]),
    ("rtod_batch_destroy", None, [_vp]),
    ("rtod_mlp_param_count", _i32, []),
    ("rtod_mlp_forward", _i32, [_i32, _vp, _vp, _i64, _vp]),
    ("rtod_mlp_grad", _i32, [_i32, _vp, _vp, _vp, _i64, _vp, _vp]),
    ("rtod_mlp_adam", _i32, [_i32, _vp, _vp, _vp, _i32, _vp, _vp, _i64, ctypes.c_float, _vp]),
    ("rtod_destroy", None, [_vp]),
    ("rtod_last_error", ctypes.c_char_p, []),
    ("rtod_version", ctypes.c_char_p, []),
]


def lib():
    """The loaded library. Raises if librtod.so is absent: the detector has no
    CPU fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m rtod_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != RTOD_OK:
        raise RtodError(code, lib().rtod_last_error().decode())
