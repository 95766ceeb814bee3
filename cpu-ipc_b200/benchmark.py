#!/usr/bin/env python3
"""Repeated independent runs of the headless GPU runner (the counterpart of
the reference's scripts/benchmark.py:54-97): each repeat is a fresh process
writing its own metrics.csv; the wall time of a run is the sum of its
step_ms column, and the summary gives the median, minimum and maximum over
the repeats.

    python cpu-ipc_b200/benchmark.py --scene cloth-drape --steps 20 --repeats 5 \\
        --precision mixed --precond learned
"""
import argparse
import csv
import statistics
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description="Benchmark the headless GPU runner over independent processes")
    ap.add_argument("--exe", type=Path, default=HERE / "cipc_headless_gpu")
    ap.add_argument("--repeats", type=int, default=5)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--scene", choices=("cloth-drape", "two-cubes", "cloth-bunny", "twisting-mat", "twisting-mat-soft", "bunny2"),
                    default="twisting-mat-soft")
    ap.add_argument("--assets", type=Path, default=None, help="Assets directory of the reference's scenes")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--precond", choices=("jacobi", "learned", "fsai"), default="jacobi")
    ap.add_argument("--output", type=Path, default=Path("Output/benchmark"))
    return ap.parse_args(argv)


def read_metrics(path):
    with path.open(newline="", encoding="utf-8") as stream:
        rows = list(csv.DictReader(stream))
    if not rows:
        raise RuntimeError(f"no metrics found in {path}")
    return rows


def run(args):
    if args.repeats <= 0 or args.steps <= 0:
        raise SystemExit("--repeats/--steps must be positive")
    samples = []
    for repeat in range(args.repeats):
        out = (args.output / f"run_{repeat + 1:02d}").resolve()
        cmd = [str(args.exe.resolve()), "--scene", args.scene, "--steps", str(args.steps), "--output", str(out),
               "--linear-solver", "gpu-pcg", "--precision", args.precision, "--precond", args.precond]
        if args.assets is not None:
            cmd += ["--assets", str(args.assets)]
        done = subprocess.run(cmd, check=True, text=True, capture_output=True)
        result = [ln for ln in done.stdout.splitlines() if ln.startswith("RESULT ")]
        if len(result) != 1:
            raise RuntimeError(f"unexpected runner output:\n{done.stdout}")
        rows = read_metrics(out / "metrics.csv")
        samples.append(sum(float(r["step_ms"]) for r in rows))
        print(f"run {repeat + 1}: {samples[-1]:.3f} ms | {result[0]}", flush=True)
    print(f"summary: median={statistics.median(samples):.3f} ms, min={min(samples):.3f} ms, max={max(samples):.3f} ms, "
          f"repeats={len(samples)}, steps={args.steps}", flush=True)
    return samples


if __name__ == "__main__":
    run(parse_args())
