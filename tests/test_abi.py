"""C-ABI checks that need no GPU: the library loads, exports every function
declared in include/rtod.h, and rejects bad input without touching a device."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "rtod.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rtod_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def native():
    from rtod_b200 import build
    build.build()
    from rtod_b200 import _native
    return _native


def test_header_declares_api():
    names = header_functions()
    for fn in ("rtod_create", "rtod_push_slide", "rtod_detect", "rtod_run", "rtod_destroy",
               "rtod_last_error"):
        assert fn in names


def test_library_exports_every_header_symbol(native):
    L = native.lib()
    for fn in header_functions():
        assert hasattr(L, fn), f"{fn} declared in include/rtod.h but not exported"
    bound = {name for name, _, _ in native.SIGNATURES}
    assert set(header_functions()) <= bound


def test_config_init_and_validation_without_gpu(native):
    L = native.lib()
    cfg = native.Config()
    assert L.rtod_config_init(ctypes.byref(cfg)) == 0
    assert (cfg.window, cfg.slide, cfg.K, cfg.dim, cfg.opt) == (100000, 5000, 50, 1, 2)
    h = ctypes.c_void_p()
    bad = native.Config()
    L.rtod_config_init(ctypes.byref(bad))
    bad.slide = 3000  # W % S != 0
    assert L.rtod_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    assert b"slide" in L.rtod_last_error()
    bad.slide, bad.dim = 5000, 9
    assert L.rtod_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad.dim, bad.R = 1, -1.0
    assert L.rtod_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    assert L.rtod_create(None, ctypes.byref(h)) == -2
    assert L.rtod_version().startswith(b"rtod-b200")
