"""The optixScan-compatible command line: flags, text formats and report."""
import numpy as np
import pytest

from rtod_b200 import cli


def test_flags_match_reference_surface():
    ap = cli.build_parser()
    a = ap.parse_args(["--n", "1048572", "--R", "0.45", "--K", "50", "--window", "100000",
                       "--slide", "5000", "-f", "x.txt", "--start_copy_pos", "2",
                       "--launch_ray_num", "7"])
    assert (a.n, a.R, a.K, a.window, a.slide, a.file, a.start_copy_pos) == (
        1048572, 0.45, 50, 100000, 5000, "x.txt", 2)
    assert a.opt == 2 and a.warmup == 10 and a.max_slides == 10000


def test_read_text_1d_and_3d(tmp_path):
    p1 = tmp_path / "s.txt"
    p1.write_text("1.5\n-2.25\n3\n4e-3\n")
    x = cli.read_text(str(p1), 3, 1)
    np.testing.assert_array_equal(x[:, 0], np.array([1.5, -2.25, 3.0], np.float32))
    p3 = tmp_path / "t.txt"
    p3.write_text("1,2,3\n4,5,6\n")
    y = cli.read_text(str(p3), 10, 3)
    assert y.shape == (2, 3) and y[1, 2] == 6.0


@pytest.mark.gpu
def test_cli_report_and_outliers(tmp_path, capsys, oracle_mod):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rtod_b200 import datagen
    pts = datagen.random_walk(6000, 0.1, seed=3)
    f = tmp_path / "walk.txt"
    f.write_text("\n".join(repr(float(v)) for v in pts[:, 0]) + "\n")
    rc = cli.main(["--n", "6000", "--R", "0.2", "--K", "8", "--window", "2000", "--slide", "200",
                   "-f", str(f), "--warmup", "1", "--print-outliers"])
    assert rc == 0
    out = capsys.readouterr().out
    for key in ("[Time] copy new points h2d", "[Time] prepare cell", "[Time] build BVH",
                "[Time] detect outlier", "[Time] total time for a slide", "BVH Node / slide",
                "[Mem] Device memory used for data(MB)", "Window size: 2000"):
        assert key in out
    off, ids, _ = oracle_mod.detect(pts, 2000, 200, 0.2, 8)
    lines = [l for l in out.splitlines() if l.startswith("slide ")]
    assert len(lines) == len(off) - 1
    for j, line in enumerate(lines):
        got = [int(t) for t in line.split(":", 1)[1].split()]
        assert got == ids[off[j]:off[j + 1]].tolist()


@pytest.mark.parametrize("dataset", ["stk", "gau", "tao"])
@pytest.mark.parametrize("param", ["window", "slide", "R", "K"])
def test_sweep_grids_follow_the_reference_driver(dataset, param):
    """Five settings per parameter, as script/run.py:76-218 varies them; every
    window a whole number of slides."""
    from rtod_b200 import sweep
    w, grid = sweep.settings(dataset, param)
    assert len(grid) == 5
    for st in grid:
        assert st["window"] % st["slide"] == 0 and st["R"] > 0 and st["K"] > 0
    assert len({tuple(sorted(st.items())) for st in grid}) == 5


@pytest.mark.gpu
def test_sweep_rows_match_oracle(oracle_mod):
    """A K sweep on the sensor-like stream, 3 slides per setting: each row's
    outliers per slide equal the oracle's for that setting."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rtod_b200 import sweep
    rows = sweep.run("tao", "K", warmup=0, max_slides=3)
    w, grid = sweep.settings("tao", "K")
    assert [r["K"] for r in rows] == [st["K"] for st in grid]
    for r in rows:
        assert r["slides"] == 3 and r["ms_per_slide"] > 0
        pts = w.points[:r["window"] + 3 * r["slide"]]
        off, ids, _ = oracle_mod.detect(pts, r["window"], r["slide"], r["R"], r["K"], "fp32_le",
                                        engine="grid", threads=8)
        assert r["outliers_per_slide"] == pytest.approx(len(ids) / 3)


def write_stream(path, pts):
    """RTOD's text format: one value per line in 1-d, x,y,z otherwise, with
    enough digits that every double (and float32) reads back exactly."""
    pts = np.asarray(pts, np.float64)
    with open(path, "w") as f:
        for row in pts:
            f.write(",".join("%.17g" % v for v in row) + "\n")


def parse_outliers(text):
    rows = [l for l in text.splitlines() if l.startswith("slide ")]
    return [[int(t) for t in l.split(":", 1)[1].split()] for l in rows]


@pytest.mark.gpu
def test_cli_double_input_bit_exact(tmp_path, capsys):
    """--coord f64: RTOD's %lf input reaches the double detector without a
    float32 cast; the double fixtures' outliers come out bit for bit."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from conftest import golden_cases_f64, load_golden
    for path in golden_cases_f64():
        meta, pts, off, ids = load_golden(path)
        f = tmp_path / "s.txt"
        write_stream(f, pts)
        rc = cli.main(["--n", str(len(pts)), "--R", repr(meta["R"]), "--K", str(meta["K"]), "--window",
                       str(meta["W"]), "--slide", str(meta["S"]), "-f", str(f), "--dim", str(pts.shape[1]),
                       "--coord", "f64", "--warmup", "1", "--print-outliers"])
        assert rc == 0
        got = parse_outliers(capsys.readouterr().out)
        assert got == [ids[off[j]:off[j + 1]].tolist() for j in range(len(off) - 1)], path


def native_cli():
    import os
    from rtod_b200 import build
    build.build()
    return os.path.join(os.path.dirname(build.LIB), "rtod")


def test_native_cli_usage():
    """The native command line (C++ over the C ABI) is built beside the
    library and rejects an incomplete command line before touching a GPU."""
    import subprocess
    r = subprocess.run([native_cli(), "--window", "10"], capture_output=True, text=True)
    assert r.returncode == 1 and "need --file" in r.stderr
    r = subprocess.run([native_cli(), "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown option '--bogus'" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["f32", "f64"])
def test_native_cli_matches_golden(tmp_path, kind):
    """rtod (C++, include/rtod.h only) on RTOD-format text files: float
    storage with the FP32 predicate against the float fixtures, double
    storage with RTOD's double test against the double fixtures."""
    import subprocess
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from conftest import golden_cases, golden_cases_f64, load_golden
    cases = golden_cases_f64() if kind == "f64" else golden_cases()
    for path in cases:
        meta, pts, off, ids = load_golden(path)
        if kind == "f32" and meta["pred"] != "fp32_le":
            continue
        f = tmp_path / "s.txt"
        write_stream(f, pts)
        # whole-stream passes (graph and not), and RTOD's per-slide loop through
        # push/detect with the grid engine and the window engine
        for extra in ([], ["--no-graph"], ["--streaming"], ["--streaming", "--engine", "window"]):
            cmd = [native_cli(), "--n", str(len(pts)), "--R", repr(meta["R"]), "--K", str(meta["K"]),
                   "--window", str(meta["W"]), "--slide", str(meta["S"]), "-f", str(f), "--dim",
                   str(pts.shape[1]), "--coord", kind, "--warmup", "1", "--print-outliers"] + extra
            r = subprocess.run(cmd, capture_output=True, text=True)
            assert r.returncode == 0, r.stderr
            assert "[Time] total time for a slide" in r.stdout and "BVH Node / slide" in r.stdout
            if "--streaming" in extra and len(off) > 2:
                assert "[Wall] slide (push + detect)" in r.stdout
            got = parse_outliers(r.stdout)
            assert got == [ids[off[j]:off[j + 1]].tolist() for j in range(len(off) - 1)], (path, extra)
