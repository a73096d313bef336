"""Generates the reference-run fixtures tests/golden/ref_*.npz: per-slide
outlier sets produced by RTOD's own code.

RTOD's host code (src/ods/optixScan.cpp: read_data, make_gas,
initialize_params, initialize_cell, detect_outlier with its FixQueue grid
filter and outlier pick) is compiled unmodified by oracle/ref/Makefile, with
its device side (the AABB kernel and the OptiX raygen / intersection
programs, src/ods/aabb.cu, src/ods/optixScan.cu:21-75, :158-199) replaced by
host stand-ins (oracle/ref/ref_fakes.cpp). Every slide is also checked by
RTOD's own brute force, check_outlier (src/ods/optixScan.cpp:817-881); a
fixture is written only when the two agree on every slide and no pair sits
at the margin where OptiX's traversal precision could decide (the float
AABB test and the double test disagree).

RTOD reads doubles (%lf) and computes in double, so these fixtures pin the
double-precision detector: RTOD_COORD_F64 storage with RTOD_PRED_F64_LT on
the GPU, and the oracle's double mode. The streams are the float32 values of
the seeded generators in rtod_b200/datagen.py (the tests regenerate them and
check a digest); the double fixtures dbl_*.npz made by make_golden.py are
run through RTOD too and must match their stored outliers.

Run (needs the RTOD sources; default /root/reference, or RTOD_REF=...):
    python tests/golden/make_ref_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import reference  # noqa: E402
from rtod_b200 import datagen  # noqa: E402  (input generation only)


def digest(pts: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(pts, np.float32).tobytes()).hexdigest()[:32]


def streams():
    """(name, generator expression, points, W, S, R, K); the expression is
    evaluated by the tests to regenerate the stream."""
    out = []
    expr = "datagen.small_walk().points"
    out.append(("ref_walk1d_W10k", expr, eval(expr), 10_000, 500, 0.45, 50))
    expr = "datagen.stock_like().points[:60_000]"
    out.append(("ref_stock1d_W20k", expr, eval(expr), 20_000, 1_000, 0.45, 50))
    expr = "datagen.gaussian_mixture(60_000, seed=3)"
    for K in (30, 70):
        out.append((f"ref_gmm1d_W10k_K{K}", expr, eval(expr), 10_000, 500, 0.028, K))
    expr = "datagen.sensor_like().points[:110_000]"
    out.append(("ref_sensor3d_W10k", expr, eval(expr), 10_000, 500, 1.9, 50))
    expr = "datagen.sensor_3d(30_000, seed=11)"
    out.append(("ref_sensor3d_W4k_K10", expr, eval(expr), 4_000, 400, 1.2, 10))
    return out


def run_one(name, pts, W, S, R, K):
    t0 = time.time()
    off, ids, boff, bids, stats = reference.detect(pts.astype(np.float64), W, S, R, K, brute=True)
    same = bool(np.array_equal(off, boff) and np.array_equal(ids, bids))
    print(f"{name}: {int(stats[2])} slides, {len(ids)} outliers, undetermined {int(stats[0])}, "
          f"margin events {int(stats[1])}, pick == brute force: {same}, {time.time() - t0:.1f} s", flush=True)
    return off, ids, stats, same


def main():
    if not reference.build():
        sys.exit("RTOD sources not found: set RTOD_REF to an RTOD checkout")
    only = set(sys.argv[1:])
    for name, expr, pts, W, S, R, K in streams():
        if only and name not in only:
            continue
        off, ids, stats, same = run_one(name, pts, W, S, R, K)
        if not same or stats[1] != 0:
            sys.exit(f"{name}: not written (pick and brute force differ, or margin events)")
        meta = {"name": name, "stream": expr, "digest": digest(pts), "W": W, "S": S, "R": R, "K": K,
                "dim": int(pts.shape[1]), "slides": int(stats[2]), "undetermined_total": int(stats[0]),
                "margin_events": int(stats[1]), "brute_force_agrees": same,
                "made_by": "RTOD src/ods/optixScan.cpp detect_outlier + check_outlier (oracle/ref)"}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), meta=np.frombuffer(json.dumps(meta).encode(), np.uint8),
                            offsets=off, ids=ids)
    # the double fixtures of make_golden.py, run through RTOD
    for path in sorted(p for p in os.listdir(HERE) if p.startswith("dbl_") and p.endswith(".npz")):
        z = np.load(os.path.join(HERE, path))
        meta = json.loads(bytes(z["meta"]).decode())
        pts = z["points"]
        if pts.shape[1] not in (1, 3):
            continue
        off, ids, boff, bids, stats = reference.detect(pts, meta["W"], meta["S"], meta["R"], meta["K"])
        agree = bool(np.array_equal(off, z["offsets"]) and np.array_equal(ids, z["ids"]))
        brute = bool(np.array_equal(boff, z["offsets"]) and np.array_equal(bids, z["ids"]))
        print(f"{path}: RTOD pick matches the fixture: {agree}; check_outlier matches: {brute}; "
              f"margin events {int(stats[1])}")


if __name__ == "__main__":
    main()
