"""The generated closed-form derivatives of the squared contact distances
(cpu-ipc_b200/csrc/distance_derivs.cuh: point-edge, point-triangle,
edge-edge and the edge-edge cross norm of the mollifier), built for the host
with nvcc and compared with the oracle's derivatives, which come from exact
second-order jets of the plain distance formulas.  No GPU: the barrier
kernels run this same code, and their parity on the device is covered by
test_gpu_parity.py."""
import ctypes as C
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "cpu-ipc_b200", "csrc")
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))

import oracle  # noqa: E402

dp = C.POINTER(C.c_double)
KINDS = {"PE": (1, 3), "PT": (2, 4), "EE": (3, 4), "EECross": (4, 4)}


@pytest.fixture(scope="module")
def dd():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tempfile.mkdtemp()
    so = os.path.join(d, "libdd.so")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-I", SRC, "-o", so,
                    os.path.join(HERE, "device_math_harness.cu")], check=True)
    L = C.CDLL(so)
    L.dd_grad_hess.restype = C.c_int
    L.dd_grad_hess.argtypes = [C.c_int, dp, dp, dp]
    return L


def _oracle(kind, pts):
    n = 3 * len(pts)
    g, H = np.zeros(n), np.zeros(n * n)
    L = oracle.lib()
    p = np.ascontiguousarray(pts, np.float64).reshape(-1)
    L.cipc_oracle_distance(kind, p.ctypes.data_as(dp), g.ctypes.data_as(dp), H.ctypes.data_as(dp))
    return g, H.reshape(n, n)


@pytest.mark.parametrize("name", list(KINDS))
def test_generated_derivatives_match_the_oracle(dd, name):
    kind, npts = KINDS[name]
    rng = np.random.default_rng(kind)
    worst_g = worst_h = 0.0
    for trial in range(200):
        # generic configurations over several length scales
        pts = rng.standard_normal((npts, 3)) * 10.0 ** rng.uniform(-3, 1)
        n = 3 * npts
        v = np.ascontiguousarray(pts.reshape(-1))
        g, H = np.zeros(n), np.zeros(n * n)
        assert dd.dd_grad_hess(kind, v.ctypes.data_as(dp), g.ctypes.data_as(dp), H.ctypes.data_as(dp)) == n
        go, Ho = _oracle(kind, pts)
        worst_g = max(worst_g, np.abs(g - go).max() / np.abs(go).max())
        worst_h = max(worst_h, np.abs(H.reshape(n, n) - Ho).max() / np.abs(Ho).max())
    assert worst_g <= 1e-10, worst_g
    assert worst_h <= 1e-9, worst_h
