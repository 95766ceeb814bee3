"""cpu-ipc_b200/benchmark.py on the host: repeated independent runs of a
runner, one metrics.csv per run, the median over the runs.  A stand-in
runner (a small script that writes the runner's files) takes the place of
the GPU binary here; the GPU runner itself is exercised by
test_gpu_headless.py."""
import os
import stat
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "cpu-ipc_b200"))
import benchmark  # noqa: E402

FAKE = """#!{py}
import os, sys
a = sys.argv
out = a[a.index("--output") + 1]
steps = int(a[a.index("--steps") + 1])
os.makedirs(out, exist_ok=True)
n = len([d for d in os.listdir(os.path.dirname(out)) if d.startswith("run_")])
with open(os.path.join(out, "metrics.csv"), "w") as f:
    f.write("frame,step_ms\\n")
    for k in range(steps):
        f.write(f"{{k}},{{10.0 * n + k}}\\n")
print("RESULT steps=%d vertices=1 sum_x=0" % steps)
"""


def test_median_over_independent_runs(tmp_path, capsys):
    exe = tmp_path / "runner"
    exe.write_text(FAKE.format(py=sys.executable))
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    args = benchmark.parse_args(["--exe", str(exe), "--repeats", "3", "--steps", "2", "--output", str(tmp_path / "out")])
    samples = benchmark.run(args)
    # run k (1-based) writes step times 10k and 10k + 1
    assert samples == [21.0, 41.0, 61.0]
    out = capsys.readouterr().out
    assert "summary: median=41.000 ms, min=21.000 ms, max=61.000 ms, repeats=3, steps=2" in out


def test_rejects_non_positive_counts(tmp_path):
    with pytest.raises(SystemExit):
        benchmark.run(benchmark.parse_args(["--repeats", "0"]))
