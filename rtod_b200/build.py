"""Builds the native library rtod_b200/librtod.so with nvcc for sm_100a.

The library is plain CUDA C++ with a C ABI (include/rtod.h); nothing in it
depends on PyTorch. Usage: ``python -m rtod_b200.build [--verbose]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "librtod.so")
CLI = os.path.join(PKG, "rtod")  # native optixScan-compatible command line (rtod_cli.cpp)
SOURCES = ["rtod.cu", "fused_f32.cu", "fused_f64.cu", "grid.cu"]
HEADERS = ["kernels.cuh", "router.cuh", "span.cuh", "group.cuh", "fused.cuh", "fused_impl.cuh", "grid.cuh"]
OBJ_DIR = os.path.join(PKG, "_build")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-fvisibility=hidden"]


def compile_command(src: str, ptxas_verbose: bool = False) -> list[str]:
    """nvcc of one translation unit to an object in OBJ_DIR."""
    cmd = [nvcc()] + FLAGS + ["-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src),
                              "-o", os.path.join(OBJ_DIR, src[:-3] + ".o")]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    return cmd


def command(out: str = LIB) -> list[str]:
    """Link of the objects into the shared library."""
    return [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", out] + \
        [os.path.join(OBJ_DIR, s[:-3] + ".o") for s in SOURCES]


def stale(out: str = LIB) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "rtod.h"))
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def cli_command() -> list[str]:
    """The native command line: plain C++ against the C ABI, linked to
    librtod.so beside it."""
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    return [cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", CLI,
            os.path.join(CSRC, "rtod_cli.cpp"), "-L", PKG, "-lrtod", "-Wl,-rpath,$ORIGIN"]


def build(force: bool = False, verbose: bool = False) -> str:
    if force or stale():
        # the translation units compile in parallel (the fused pipeline's
        # instantiations are about as large as the rest of the library)
        os.makedirs(OBJ_DIR, exist_ok=True)
        procs = [subprocess.Popen(compile_command(src, verbose), stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                  text=True) for src in SOURCES]
        outs = [p.communicate()[0] for p in procs]
        for p, o in zip(procs, outs):
            if p.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + o)
        if verbose:
            sys.stdout.write("".join(outs))
        r = subprocess.run(command(), capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    cli_src = os.path.join(CSRC, "rtod_cli.cpp")
    if force or not os.path.exists(CLI) or os.path.getmtime(CLI) < max(os.path.getmtime(LIB),
                                                                          os.path.getmtime(cli_src)):
        r = subprocess.run(cli_command(), capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("building the rtod command line failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))
