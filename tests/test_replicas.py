"""The multi-rank path of bench.py on host ranks (gloo, world size 2, no GPU):
the replica plumbing (barriers, maximum of the timed durations over ranks,
whole-job value, rank 0 alone printing) and the reference arm under
torchrun, whose other ranks exit without work. The detector itself has no
collective: ranks are independent replicas."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun(args, n=2, timeout=300):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), "bench.py"] + args
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout, env=env)
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    return p, lines


def test_replica_plumbing_two_ranks():
    p, lines = torchrun(["--mode", "replica-check"])
    assert p.returncode == 0, p.stderr[-2000:]
    assert len(lines) == 1, p.stdout  # rank 0 alone prints
    r = json.loads(lines[0])
    assert r["n_ranks"] == 2 and r["identical_on_all_ranks"] is True
    assert r["value"] > 0 and r["s_max"] > 0 and r["outliers"] > 0


def test_reference_arm_two_ranks():
    p, lines = torchrun(["--impl", "reference", "--steps", "1", "--warmup", "0"])
    assert p.returncode == 0, p.stderr[-2000:]
    assert len(lines) == 1, p.stdout
    r = json.loads(lines[0])
    assert r["impl"] == "reference" and r["n_gpus"] == 2
    assert r["e2e"]["h2d_bytes_per_step"] == 0 and r["cpu_baseline"]["kind"] == "port"
