"""rtod_b200: sliding-window distance outlier detection on NVIDIA B200 (sm_100a).

A drop-in for the per-slide detector of RTOD (Wang-Zm/rtod): same run
surface (window, slide, R, K, dimension, optimisation level, per-slide
outlier IDs, per-stage times), with the OptiX/RT-core path replaced by
hand-written CUDA kernels behind the C ABI in include/rtod.h.
"""
from ._native import RtodError  # noqa: F401
from .engine import BatchDetector, Detector, RunResult  # noqa: F401

__all__ = ["Detector", "BatchDetector", "RunResult", "RtodError"]
