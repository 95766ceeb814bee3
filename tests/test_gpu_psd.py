"""PSD projection of the contact Hessians on a B200: the half-warp one-sided
Jacobi sweep in registers (halfWarpPsdProject12, used by the self-contact
barrier kernel) and the warp shared-memory two-sided sweep (warpPsdProject,
the mollified edge-edge and hinge kernels),
both against numpy's eigen-decomposition V max(L, 0) V^T, which is the rule
of the reference's makePD (CPU IPC/IPCSolver.cpp:238-267).

Cases: random indefinite matrices over twelve orders of magnitude, barrier-like
matrices ca g g^T + cb H with cb < 0, positive definite matrices (returned
unchanged, bit for bit), contacts of 2 and 3 points zero-padded to 12 (the
padding stays zero), matrices with repeated eigenvalues, and an odd count so
that the last half warp has no matrix."""
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

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def project():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    d = tempfile.mkdtemp()
    so = os.path.join(d, "libpsd.so")
    subprocess.run([nvcc, "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", SRC, "-o", so, os.path.join(HERE, "psd_harness.cu")], check=True)
    L = C.CDLL(so)
    L.psd12_project.argtypes = [C.c_int, C.c_int, dp, dp]
    L.psd12_project.restype = C.c_int

    def run(which, A):
        A = np.ascontiguousarray(A, np.float64)
        out = np.zeros_like(A)
        caps = L.psd12_project(which, A.shape[0], A.ctypes.data_as(dp), out.ctypes.data_as(dp))
        assert caps == 0, caps
        return out
    return run


def reference_projection(A):
    w, V = np.linalg.eigh(A)
    if w.min() >= 0:
        return A.copy()
    return (V * np.maximum(w, 0)) @ V.T


def cases(seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(120):  # indefinite, scales 1e-6 .. 1e6
        B = rng.standard_normal((12, 12)) * 10.0 ** rng.uniform(-6, 6)
        out.append(B + B.T)
    for k in range(120):  # barrier-like: b'' g g^T + b' H with b' < 0
        g = rng.standard_normal(12)
        H = rng.standard_normal((12, 12))
        out.append(rng.uniform(1, 1e4) * np.outer(g, g) - rng.uniform(0.1, 10) * (H + H.T))
    for k in range(40):  # positive definite
        B = rng.standard_normal((12, 12))
        out.append(B @ B.T + 1e-3 * np.eye(12))
    for nd in (6, 9):  # point-point and point-edge contacts, zero-padded
        for k in range(40):
            B = rng.standard_normal((nd, nd))
            A = np.zeros((12, 12))
            A[:nd, :nd] = B + B.T
            out.append(A)
    for k in range(20):  # repeated eigenvalues
        Q, _ = np.linalg.qr(rng.standard_normal((12, 12)))
        lam = np.repeat(rng.standard_normal(4), 3)
        out.append((Q * lam) @ Q.T)
    return np.stack(out)


@pytest.mark.parametrize("which", [0, 1])
def test_projection_matches_eigen_decomposition(project, which):
    A = cases()
    n = A.shape[0] - 1  # odd: the last half warp is idle
    A = A[:n]
    P = project(which, A.reshape(n, 144)).reshape(n, 12, 12)
    for i in range(n):
        R = reference_projection(A[i])
        scale = np.linalg.norm(A[i])
        assert np.max(np.abs(P[i] - R)) <= 1e-12 * scale, (which, i, np.max(np.abs(P[i] - R)) / scale)
        assert np.linalg.eigvalsh(0.5 * (P[i] + P[i].T)).min() >= -1e-12 * scale


def test_register_sweep_details(project):
    A = cases(1)
    n = A.shape[0]
    P = project(0, A.reshape(n, 144)).reshape(n, 12, 12)
    for i in range(n):
        if np.linalg.eigvalsh(A[i]).min() > 1e-9 * np.linalg.norm(A[i]):
            # no negative eigenvalue: the input comes back unchanged, bit for bit
            assert np.array_equal(P[i], A[i]), i
        else:
            # a projected matrix is exactly symmetric
            assert np.array_equal(P[i], P[i].T), i
        nz = np.flatnonzero(np.abs(A[i]).sum(axis=0))
        pad = np.setdiff1d(np.arange(12), nz)
        if pad.size:
            assert not np.any(P[i][pad, :]) and not np.any(P[i][:, pad]), i
    # both sweeps agree
    W = project(1, A.reshape(n, 144)).reshape(n, 12, 12)
    for i in range(n):
        assert np.max(np.abs(P[i] - W[i])) <= 1e-12 * np.linalg.norm(A[i]), i
