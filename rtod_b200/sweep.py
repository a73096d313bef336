"""Parameter sweeps of RTOD's experiment driver on synthetic streams.

Mirrors the grids of ``*_vary_parameters`` in script/run.py:76-218: window
sizes {10k, 50k, 100k, 150k, 200k} (S = 5k), slide as a fraction of the
window {5%, 10%, 20%, 50%, 100%} (W = 100k), R scaled by {0.25, 0.5, 1, 5,
10} and K in {10, 30, 50, 70, 100}, for the GAU and STK stand-ins (W values
for TAO are 1k..20k with S = 500, R = 1.9). Each setting runs one timed pass
after warm-up and prints the per-slide time, like the reference's logs.

    python -m rtod_b200.sweep --dataset stk --param K
"""
from __future__ import annotations

import argparse
import json
import sys

from . import datagen
from .engine import Detector

GRIDS = {
    "stk": dict(make=datagen.stock_like, windows=[10_000, 50_000, 100_000, 150_000, 200_000], S=5_000),
    "gau": dict(make=datagen.gaussian_like, windows=[10_000, 50_000, 100_000, 150_000, 200_000], S=5_000),
    "tao": dict(make=datagen.sensor_like, windows=[1_000, 5_000, 10_000, 15_000, 20_000], S=500),
}
SLIDE_FRACS = [0.05, 0.1, 0.2, 0.5, 1.0]
R_SCALES = [0.25, 0.5, 1.0, 5.0, 10.0]
K_LIST = [10, 30, 50, 70, 100]


def settings(dataset: str, param: str):
    g = GRIDS[dataset]
    w = g["make"]()
    base = dict(window=w.window, slide=w.slide, R=w.R, K=w.K)
    if param == "window":
        return w, [dict(base, window=W, slide=g["S"]) for W in g["windows"]]
    if param == "slide":
        return w, [dict(base, slide=int(w.window * f)) for f in SLIDE_FRACS]
    if param == "R":
        return w, [dict(base, R=w.R * f) for f in R_SCALES]
    if param == "K":
        return w, [dict(base, K=k) for k in K_LIST]
    raise ValueError(param)


def run(dataset: str, param: str, warmup: int = 2, router: bool = False, tuner: bool = False,
        max_slides: int = 10000):
    w, grid = settings(dataset, param)
    rows = []
    for st in grid:
        with Detector(st["window"], st["slide"], st["R"], st["K"], dim=w.dim, router=router,
                      tuner=tuner) as det:
            for _ in range(warmup):
                det.reset()
                det.run(w.points, max_slides=max_slides)
            det.reset()
            res = det.run(w.points, max_slides=max_slides, times=True)
        rows.append(dict(st, dataset=dataset, slides=res.slides, ms_per_slide=res.times["total"],
                         outliers_per_slide=float(res.offsets[-1]) / max(1, res.slides),
                         undetermined_per_slide=res.times["undetermined_per_slide"]))
    return rows


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--dataset", choices=sorted(GRIDS), default="stk")
    ap.add_argument("--param", choices=["window", "slide", "R", "K"], default="K")
    ap.add_argument("--router", action="store_true", help="learned router on (window engine)")
    ap.add_argument("--tuner", action="store_true", help="autotune each setting on its first slides")
    ap.add_argument("--max-slides", type=int, default=10000, help="slides per pass (RTOD caps at 10000)")
    ap.add_argument("--warmup", type=int, default=2)
    args = ap.parse_args(argv)
    for row in run(args.dataset, args.param, warmup=args.warmup, router=args.router, tuner=args.tuner,
                   max_slides=args.max_slides):
        print(json.dumps(row))
    return 0


if __name__ == "__main__":
    sys.exit(main())
