"""Builds libcipc_gpu.so (the C-ABI library) from csrc/ for sm_100a.

Usage: python build.py [--jobs N] [--force]

Every CUDA file is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``; the collision unit is
compiled with ``--fmad=false`` so that box overlaps, closest-feature
classification and distance thresholds round exactly like the FP64 oracle.
The host-only set-up file is compiled by g++.  Outputs land in _build/ and
the shared library beside this file, with the headless runner
(apps/cipc_headless_gpu.cpp, linked against the library) next to it.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcipc_gpu.so")
HEADLESS_SRC = os.path.join(HERE, "apps", "cipc_headless_gpu.cpp")
HEADLESS = os.path.join(HERE, "cipc_headless_gpu")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", SRC,
          "-I", os.path.join(HERE, "..", "include")]
UNITS = {
    "elastic.cu": [],
    "collision.cu": ["--fmad=false"],
    "contact.cu": [],
    "pcg.cu": [],
    "mpnn.cu": [],
    "fsai.cu": [],
    "util.cu": [],
    "solver.cu": [],
}
HOST_UNITS = {"scene_setup.cpp": []}


def _stale(obj, src_files):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in src_files)


def _headers():
    return [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".h", ".cuh"))] + \
        [os.path.join(HERE, "..", "include", "cipc_gpu.h")]


def compile_unit(name, extra, force):
    src = os.path.join(SRC, name)
    obj = os.path.join(OUT, name + ".o")
    if not force and not _stale(obj, [src] + _headers()):
        return obj, None
    if name.endswith(".cu"):
        cmd = [NVCC] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
    else:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-I", SRC, "-c", src, "-o", obj] + extra
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "$ " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, None


def build(jobs=8, force=False):
    os.makedirs(OUT, exist_ok=True)
    units = list(UNITS.items()) + list(HOST_UNITS.items())
    objs, errors = [], []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(compile_unit, n, e, force) for n, e in units]
        for f in futs:
            obj, err = f.result()
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("compilation failed:\n" + "\n".join(errors))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    # the headless runner links only against the C ABI library
    if force or _stale(HEADLESS, [HEADLESS_SRC, os.path.join(HERE, "apps", "runtime_files.h"), LIB,
                                  os.path.join(HERE, "..", "include", "cipc_gpu.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(HERE, "..", "include"), HEADLESS_SRC, "-o", HEADLESS,
               "-L", HERE, "-lcipc_gpu", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("headless runner build failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.jobs, a.force))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
