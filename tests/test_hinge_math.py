"""The library's hinge bending element math (cpu-ipc_b200/csrc/hinge_bending.cuh:
closed-form angle gradient, forward-mode Hessian) built for the host and
compared with the oracle's element (second-order jets, makePD projection), no
GPU.  The GPU kernel (elastic.cu, hingeKernel) runs this same code; its
parity with the oracle is in test_gpu_parity.py."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "cpu-ipc_b200", "csrc")
dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def harness():
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("g++ not available")
    d = tempfile.mkdtemp()
    so = os.path.join(d, "libhinge.so")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-I", SRC, "-o", so, os.path.join(HERE, "hinge_harness.cpp")], check=True)
    L = C.CDLL(so)
    L.hinge_element.restype = C.c_double
    L.hinge_element.argtypes = [dp, dp, C.c_double, dp, dp]
    L.hinge_angle.restype = C.c_double
    L.hinge_angle.argtypes = [dp]
    L.hinge_hess_column.argtypes = [dp, C.c_int, dp]
    L.hinge_angle_hess_full.restype = C.c_double
    L.hinge_angle_hess_full.argtypes = [dp, dp]
    return L


def _element(L, x, rest, k):
    x = np.ascontiguousarray(x, np.float64).reshape(12)
    r = np.ascontiguousarray(rest, np.float64).reshape(12)
    g = np.zeros(12)
    H = np.zeros(144)
    e = L.hinge_element(x.ctypes.data_as(dp), r.ctypes.data_as(dp), float(k), g.ctypes.data_as(dp), H.ctypes.data_as(dp))
    return e, g, H.reshape(12, 12)


def _psd(H):
    w, V = np.linalg.eigh(0.5 * (H + H.T))
    return (V * np.maximum(w, 0.0)) @ V.T


def _shapes(rng):
    rest = np.array([[0, 0, 0], [1, 1, 0], [1, 0, 0], [0, 1, 0]], float) + 0.05 * rng.standard_normal((4, 3))
    yield rest + 0.3 * rng.standard_normal((4, 3)), rest
    # folded almost flat onto itself: theta - theta0 close to +/- pi
    folded = rest.copy()
    folded[3] = rest[2] + np.array([0.02, -0.01, 0.03])
    yield folded, rest
    # a bent rest shape
    bent = rest.copy()
    bent[3, 2] += 0.6
    yield rest + 0.1 * rng.standard_normal((4, 3)), bent


def test_hinge_math_matches_oracle(harness, oracle_mod):
    rng = np.random.default_rng(11)
    for _ in range(4):
        for x, rest in _shapes(rng):
            eo, go, Ho = oracle_mod.hinge(x, rest, 2.5)
            em, gm, Hm = _element(harness, x, rest, 2.5)
            assert abs(em - eo) <= 1e-12 * max(1.0, abs(eo))
            assert np.abs(gm - go).max() <= 1e-10 * max(1.0, np.abs(go).max())
            assert np.abs(Hm - Hm.T).max() <= 1e-10 * max(1.0, np.abs(Hm).max())
            assert np.abs(_psd(Hm) - Ho).max() <= 1e-9 * max(1.0, np.abs(Ho).max())


def test_hinge_angle_is_zero_flat_and_odd_under_swapping_sides(harness):
    x = np.array([[0, 0, 0], [1, 0, 0], [0.3, 1, 0], [0.6, -1, 0]], float)
    assert abs(harness.hinge_angle(np.ascontiguousarray(x.reshape(12)).ctypes.data_as(dp))) < 1e-15
    x[2, 2] = 0.4
    a = harness.hinge_angle(np.ascontiguousarray(x.reshape(12)).ctypes.data_as(dp))
    b = harness.hinge_angle(np.ascontiguousarray(x[[0, 1, 3, 2]].reshape(12)).ctypes.data_as(dp))
    assert abs(a + b) < 1e-14 and abs(a) > 0.1


def test_hinge_hessian_columns_one_direction_at_a_time(harness):
    """The one-direction form (a lane per Hessian column on the GPU) gives the
    same hess(theta) as the 12-direction form."""
    rng = np.random.default_rng(3)
    x = (np.array([[0, 0, 0], [1, 1, 0], [1, 0, 0], [0, 1, 0]], float) + 0.2 * rng.standard_normal((4, 3))).reshape(12)
    x = np.ascontiguousarray(x)
    full = np.zeros(144)
    harness.hinge_angle_hess_full(x.ctypes.data_as(dp), full.ctypes.data_as(dp))
    full = full.reshape(12, 12)
    cols = np.zeros((12, 12))
    for j in range(12):
        c = np.zeros(12)
        harness.hinge_hess_column(x.ctypes.data_as(dp), j, c.ctypes.data_as(dp))
        cols[:, j] = c
    assert np.abs(cols - full).max() <= 1e-12 * np.abs(full).max()
