"""Command line with the run surface of RTOD's ``optixScan``.

    python -m rtod_b200.cli --n 1048572 --R 0.45 --K 50 --window 100000 --slide 5000 -f stock.txt

Flags follow ``parse_args`` (src/ods/optixScan.cpp:149-212): ``--file/-f``,
``--n``, ``--window``, ``--slide``, ``--R``, ``--K``, ``--start_copy_pos``,
``--launch_ray_num`` (accepted; it only sizes RTOD's OPTIMIZATION=0 ray
launch and has no effect here). RTOD's compile-time switches become flags:
``--dim`` (DIMENSION, optixScan.h:10-12) and ``--opt`` (OPTIMIZATION,
optixScan.h:22-24). Input text is parsed like ``read_data``
(optixScan.cpp:95-147): one value per line in 1-d, ``x,y,z`` (comma
separated) otherwise, as doubles. ``--coord f64`` keeps those doubles end to
end and compares them with RTOD's double predicate (RTOD's own arithmetic,
bit for bit); the default stores float32 and uses the FP32 predicate. ``--synthetic NAME`` uses a built-in stand-in stream
instead of a file. The report mirrors RTOD's stdout (``DIM[i]``, the common
info block of optixScan.cpp:934-945, the ``[Time]`` block of
src/ods/timer.h:102-117, ``[Mem]`` lines and ``BVH Node / slide``).
Timing follows main() (optixScan.cpp:1159-1168): ``--warmup`` untimed passes
over the whole stream (RTOD: 10), then one timed pass, averaged per slide.
A graph-replayed pass measures the total only; its stage split comes from a
diagnostic pass on the same handle (each kernel launched on its own with
CUDA events) and is labelled as such. ``rtod_b200/rtod`` is the same
command line as a native C++ program.
"""
from __future__ import annotations

import argparse
import resource
import sys

import numpy as np

from . import datagen
from .engine import Detector

SYNTHETIC = {
    "walk": datagen.small_walk,
    "stk": datagen.stock_like,
    "tao": datagen.sensor_like,
    "gau": datagen.gaussian_like,
}


def read_text(path: str, n: int, dim: int, f64: bool = False) -> np.ndarray:
    """First n rows of a text stream: `%lf` per line (1-d) or comma-separated
    values (dim > 1), parsed as float64; float32 unless f64."""
    try:
        import pandas as pd
        df = pd.read_csv(path, header=None, nrows=n, sep=",", dtype=np.float64, engine="c")
        arr = df.to_numpy()
    except ImportError:  # pragma: no cover - pandas is part of the image
        arr = np.loadtxt(path, delimiter=",", max_rows=n, dtype=np.float64, ndmin=2)
    if arr.shape[1] < dim:
        raise ValueError(f"{path}: rows have {arr.shape[1]} values, need {dim}")
    return np.ascontiguousarray(arr[:, :dim], dtype=np.float64 if f64 else np.float32)


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="rtod", description=__doc__.split("\n")[0],
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--file", "-f", dest="file", default=None)
    ap.add_argument("--n", type=int, default=int(1e8), help="data num; defaults to 1e8")
    ap.add_argument("--window", type=int, default=None)
    ap.add_argument("--slide", type=int, default=None)
    ap.add_argument("--R", type=float, default=None)
    ap.add_argument("--K", type=int, default=None)
    ap.add_argument("--start_copy_pos", type=int, default=0)
    ap.add_argument("--launch_ray_num", type=int, default=0)
    ap.add_argument("--dim", type=int, default=None, help="DIMENSION (1..8)")
    ap.add_argument("--opt", type=int, default=2, help="OPTIMIZATION: 0 no grid filter, 1/2 grid filter")
    ap.add_argument("--pred", choices=["fp32_le", "f64_lt"], default=None,
                    help="neighbour test (default fp32_le; f64_lt with --coord f64)")
    ap.add_argument("--coord", choices=["f32", "f64"], default="f32",
                    help="f64: keep the input doubles and RTOD's double test end to end")
    ap.add_argument("--router", action="store_true", help="learned router on")
    ap.add_argument("--tuner", action="store_true", help="autotune grid and block shape")
    ap.add_argument("--no-graph", action="store_true", help="launch kernels one by one")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--max-slides", type=int, default=10000)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--synthetic", choices=sorted(SYNTHETIC), default=None)
    ap.add_argument("--print-outliers", action="store_true",
                    help="print each slide's outlier IDs (global stream indices)")
    return ap


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    if args.synthetic:
        w = SYNTHETIC[args.synthetic]()
        pts = w.points.astype(np.float64) if args.coord == "f64" else w.points
        window = args.window or w.window
        slide = args.slide or w.slide
        R = args.R if args.R is not None else w.R
        K = args.K if args.K is not None else w.K
        infile = f"<synthetic:{w.name}>"
    else:
        if not args.file or None in (args.window, args.slide, args.R, args.K):
            print("need --file, --window, --slide, --R and --K (or --synthetic)", file=sys.stderr)
            return 1
        pts = read_text(args.file, args.n, args.dim or 1, f64=args.coord == "f64")
        window, slide, R, K, infile = args.window, args.slide, args.R, args.K, args.file
    dim = args.dim or pts.shape[1]
    pts = pts[:args.n, :dim]
    for i in range(dim):
        print(f"DIM[{i}]: {pts[:, i].min():g}, {pts[:, i].max():g}")
    pts = np.ascontiguousarray(pts[args.start_copy_pos * slide:])
    pred = args.pred or ("f64_lt" if args.coord == "f64" else "fp32_le")
    rss0 = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss
    with Detector(window, slide, R, K, dim=dim, opt=args.opt, pred=pred, router=args.router,
                  tuner=args.tuner, use_graph=not args.no_graph, device=args.device,
                  coord=args.coord) as det:
        print(f"Dimension: {dim}")
        print(f"data num: {len(pts)}")
        print(f"R: {R}, R2: {R * R}")
        print(f"K: {K}")
        print(f"Window size: {window}")
        print(f"Slide size: {slide}")
        print(f"Input file: {infile}")
        print(f"Optimization: {args.opt}")
        for _ in range(args.warmup):
            det.reset()
            det.run(pts, max_slides=args.max_slides)
        det.reset()
        res = det.run(pts, max_slides=args.max_slides, times=True)
        t = dict(res.times)
        split_note = None
        if not args.no_graph and args.coord == "f32":
            # Graph replay gives the total only; the stage split comes from a
            # diagnostic pass on the same handle (kernels one by one, events).
            det.reset()
            ms = list(det.profile(pts, max_slides=args.max_slides).values())
            ms += [0.0] * (7 - len(ms))
            t["prepare_cell"] = ms[0] + ms[1]
            t["build_bvh"] = ms[2] + ms[3]
            t["detect_outlier"] = ms[4] + ms[5] + ms[6]
            split_note = ("(stage split: device time per slide of a diagnostic pass on the same handle, "
                          "kernels launched one by one; total: the graph-replayed pass)")
        print()
        print("###########   Time  ##########")
        print(f"[Time] copy new points h2d: {t['copy_new_points_h2d']:g} ms")
        print(f"[Time] copy filtered points h2d: {t['copy_filtered_points_h2d']:g} ms")
        print(f"[Time] copy outlier d2h: {t['copy_outlier_d2h']:g} ms")
        print(f"[Time] prepare cell: {t['prepare_cell']:g} ms")
        print(f"[Time] build BVH: {t['build_bvh']:g} ms")
        print(f"[Time] detect outlier: {t['detect_outlier']:g} ms")
        print(f"[Time] total time for a slide: {t['total']:g} ms")
        print("##############################")
        if split_note:
            print(split_note)
        print()
        rss1 = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss
        print(f"[Mem] Host cpu memory used(MB): {(rss1 - rss0) / 1024:g}")
        print(f"[Mem] Device memory used for data(MB): {det.stats['device_bytes'] / (1 << 20):g}")
        print(f"BVH Node / slide: {int(t['undetermined_per_slide'])}")
        print(f"Outliers / slide: {res.offsets[-1] / max(1, res.slides):g}")
        if args.print_outliers:
            for j in range(res.slides):
                ids = res.slide(j)
                print(f"slide {j}: " + " ".join(map(str, ids.tolist())))
    return 0


if __name__ == "__main__":
    sys.exit(main())
