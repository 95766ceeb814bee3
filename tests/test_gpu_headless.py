"""The headless GPU runner on a B200: a run resumed from its own checkpoint
continues the uninterrupted run (the reference's --resume, IPCSolver.cpp:
1085-1102, 1318-1332), and the repeated-runs benchmark (benchmark.py, the
counterpart of the reference's scripts/benchmark.py) reports the median of
independent processes."""
import os
import re
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "cpu-ipc_b200", "cipc_headless_gpu")
ASSETS = os.path.join(ROOT, "tests", "golden", "assets")


def _run(*args):
    r = subprocess.run([EXE, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("RESULT ")]
    assert len(line) == 1, r.stdout
    return dict(re.findall(r"(\w+)=(\S+)", line[0]))


def test_resume_continues_the_uninterrupted_run(tmp_path):
    common = ["--scene", "two-cubes", "--cells", "3", "--precision", "fp64", "--precond", "jacobi"]
    full = _run(*common, "--steps", "20", "--output", str(tmp_path / "full"))
    out = str(tmp_path / "split")
    _run(*common, "--steps", "10", "--write-checkpoints", "--output", out)
    assert os.path.isdir(os.path.join(out, "tempData"))
    resumed = _run(*common, "--steps", "10", "--resume", "--output", out)
    a, b = float(full["squared_norm_sum"]), float(resumed["squared_norm_sum"])
    assert abs(a - b) <= 1e-9 * abs(a), (a, b)
    # the resumed run appended its ten frames to the metrics it continues
    with open(os.path.join(out, "metrics.csv")) as f:
        frames = [int(ln.split(",")[0]) for ln in f.read().splitlines()[1:]]
    assert frames == list(range(20))


def test_repeated_runs_benchmark(tmp_path):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "cpu-ipc_b200", "benchmark.py"), "--scene", "twisting-mat-soft", "--assets", ASSETS,
                        "--steps", "1", "--repeats", "3", "--output", str(tmp_path)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    runs = [ln for ln in r.stdout.splitlines() if ln.startswith("run ")]
    assert len(runs) == 3
    assert "summary: median=" in r.stdout and "repeats=3" in r.stdout
