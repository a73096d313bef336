"""GPU entry points of the router network (forward, gradient, Adam step),
used to check the hand-written CUDA training kernels against a CPU
restatement. Parameter packing: W1[32][3], b1[32], W2[32][32], b2[32],
W3[4][32], b3[4]."""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import check, lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def param_count() -> int:
    return int(lib().rtod_mlp_param_count())


def forward(params, x, device: int = 0) -> np.ndarray:
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros((x.shape[0], 4), np.float32)
    check(lib().rtod_mlp_forward(device, _p(params), _p(x), x.shape[0], _p(out)))
    return out


def loss_grad(params, x, y, device: int = 0):
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    g = np.zeros(params.size, np.float32)
    loss = np.zeros(1, np.float32)
    check(lib().rtod_mlp_grad(device, _p(params), _p(x), _p(y), x.shape[0], _p(g), _p(loss)))
    return float(loss[0]), g


def adam_step(params, m, v, t, x, y, lr=1e-3, device: int = 0):
    p = np.array(params, np.float32)
    m = np.array(m, np.float32)
    v = np.array(v, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    loss = np.zeros(1, np.float32)
    check(lib().rtod_mlp_adam(device, _p(p), _p(m), _p(v), t, _p(x), _p(y), x.shape[0],
                              ctypes.c_float(lr), _p(loss)))
    return p, m, v, float(loss[0])
