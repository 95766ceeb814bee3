"""The rotation-aware 3x3 SVD of the elastic kernels (svd3 in
cpu-ipc_b200/csrc/cipc_device.cuh), built for the host with nvcc: U and V
are proper rotations, the singular values come out in descending magnitude
with the sign of det F on the last one, and U diag(s) V^T rebuilds F.  The
Neo-Hookean Hessian projection of the tetrahedron kernel is built on it.
No GPU."""
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
def svd3():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tempfile.mkdtemp()
    so = os.path.join(d, "libdm.so")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-I", SRC, "-o", so,
                    os.path.join(HERE, "device_math_harness.cu")], check=True)
    L = C.CDLL(so)
    L.svd3_host.argtypes = [dp, dp, dp, dp]

    def run(F):
        F = np.ascontiguousarray(F, np.float64).reshape(9)
        U, s, V = np.zeros(9), np.zeros(3), np.zeros(9)
        L.svd3_host(F.ctypes.data_as(dp), U.ctypes.data_as(dp), s.ctypes.data_as(dp), V.ctypes.data_as(dp))
        return U.reshape(3, 3), s, V.reshape(3, 3)
    return run


def _rotation(rng):
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    return q if np.linalg.det(q) > 0 else -q


def _cases(rng):
    for _ in range(300):  # generic, about half of them inverted
        yield rng.standard_normal((3, 3))
    for _ in range(100):  # deformation gradients near the rest shape, some inverted
        F = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        yield F if rng.random() < 0.8 else F @ np.diag([1, 1, -1])
    for sv in ([2.0, 1.0, 0.0], [1.0, 1.0, 1.0], [3.0, 3.0, 0.5], [1e3, 1.0, 1e-3]):
        for _ in range(20):  # rank-deficient, repeated and ill-conditioned spectra
            yield _rotation(rng) @ np.diag(sv) @ _rotation(rng).T


def test_svd3_rebuilds_and_orders(svd3):
    rng = np.random.default_rng(11)
    worst = 0.0
    for F in _cases(rng):
        U, s, V = svd3(F)
        for R in (U, V):
            assert np.abs(R.T @ R - np.eye(3)).max() <= 1e-12
            assert abs(np.linalg.det(R) - 1.0) <= 1e-12
        assert s[0] >= 0 and s[1] >= 0
        assert abs(s[0]) >= abs(s[1]) - 1e-12 * abs(s[0]) and abs(s[1]) >= abs(s[2]) - 1e-12 * abs(s[0])
        ref = np.linalg.svd(F, compute_uv=False)
        scale = max(ref[0], 1e-300)
        assert np.abs(np.abs(s) - ref).max() <= 1e-10 * scale
        d = np.linalg.det(F)
        if abs(d) > 1e-9 * scale ** 3:
            assert np.sign(s[2]) == np.sign(d)
        worst = max(worst, np.abs(U @ np.diag(s) @ V.T - F).max() / scale)
    assert worst <= 1e-10, worst
