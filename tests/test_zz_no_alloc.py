"""The allocation-free PCG entry point (cipc_gpu_pcg_bsr_noalloc).

Some callers cannot allocate device memory at solve time: a host whose GPU
memory is owned by its own allocator (here PyTorch's caching allocator owns
the matrix, right-hand side and solution), or a loop that must not pay
cudaMalloc latency.  This entry point takes device buffers from the caller and
keeps its scratch in a fixed array inside the library.  The test calls it
through the C ABI twice in a row and checks each result against the
allocating entry point, within the residual tolerance the other PCG tests
use.  It runs last so that a failure here cannot hide other failures.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import cipc

pytestmark = pytest.mark.gpu


def _spd_block_system(nv=400, seed=0):
    rng = np.random.default_rng(seed)
    blocks = {}
    for i in range(nv):
        for j in (i, (i + 1) % nv, (i + 11) % nv):
            B = rng.standard_normal((3, 3)) * 0.1
            blocks.setdefault((i, j), np.zeros((3, 3)))
            blocks[(i, j)] += B
            blocks.setdefault((j, i), np.zeros((3, 3)))
            blocks[(j, i)] += B.T
    for i in range(nv):
        blocks[(i, i)] += 4.0 * np.eye(3)
    keys = sorted(blocks)
    rp = np.zeros(nv + 1, np.int32)
    for (i, _) in keys:
        rp[i + 1] += 1
    rp = np.cumsum(rp).astype(np.int32)
    ci = np.array([j for (_, j) in keys], np.int32)
    vals = np.ascontiguousarray(np.stack([blocks[k] for k in keys]))
    b = rng.standard_normal(3 * nv)
    A = sp.bsr_matrix((vals, ci, rp), shape=(3 * nv, 3 * nv)).tocsr()
    return rp, ci, vals, b, A


def test_noalloc_pcg_matches_allocating_entry_point():
    import torch

    torch.cuda.set_device(0)
    rp, ci, vals, b, A = _spd_block_system()
    nv = len(rp) - 1
    tol = 1e-8
    x_ref, it_ref, _ = cipc.pcg_bsr(rp, ci, vals, b, precision="fp64", tol=tol)
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(rp).to(dev)
    d_ci = torch.from_numpy(ci).to(dev)
    d_vals = torch.from_numpy(vals.reshape(-1)).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    L = cipc.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        d_sol = torch.full((3 * nv,), float("nan"), dtype=torch.float64, device=dev)
        it = C.c_int(0)
        rr = C.c_double(0)
        rc = L.cipc_gpu_pcg_bsr_noalloc(nv, d_rp.data_ptr(), d_ci.data_ptr(), d_vals.data_ptr(), d_b.data_ptr(), d_sol.data_ptr(),
                                        tol, 10000, C.c_void_p(stream), C.byref(it), C.byref(rr))
        torch.cuda.synchronize()
        assert rc == 0, f"call {call}: rc {rc}"
        x = d_sol.cpu().numpy()
        assert np.linalg.norm(A @ x - b) <= 1e-6 * np.linalg.norm(b)
        assert it.value == it_ref
        assert np.allclose(x, x_ref, rtol=1e-9, atol=1e-12 * np.abs(x_ref).max())


def test_noalloc_rejects_oversized_systems():
    L = cipc.lib()
    it = C.c_int(0)
    rr = C.c_double(0)
    rc = L.cipc_gpu_pcg_bsr_noalloc(cipc.NOALLOC_MAX_ROWS + 1, 1, 1, 1, 1, 1, 1e-6, 100, None, C.byref(it), C.byref(rr))
    assert rc == 1
